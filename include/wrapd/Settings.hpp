/* Settings.hpp -- wrapd::Settings (the reference's src/Settings.hpp:29-165 and
 * its parse_args, src/Settings.cpp:31-176): the solver's flags with the
 * reference's defaults and the reference's command-line syntax (a token that
 * starts with '-' and not with a digit or '.' opens a flag; the tokens after
 * it are its value).  Extensions, after the reference's flags: -youngs E,
 * -lbfgs_m M, -rw_every N, -precision fp64|mixed, -prox lbfgs|newton, -leaf N,
 * -device D, -autotune 0|1 (the fields of wrapd_settings in ../wrapd_gpu.h).
 * One difference: should_save_data() starts true (the reference leaves it
 * uninitialised until -s is given).  See Math.hpp for this directory. */
#ifndef WRAPD_COMPAT_SETTINGS_HPP
#define WRAPD_COMPAT_SETTINGS_HPP

#include <filesystem>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../wrapd_gpu.h"
#include "Math.hpp"
#include "ModelSettings.hpp"

namespace wrapd {

struct Settings {
    class IO {
    public:
        std::string rest_mesh() const { return m_rest_mesh; }
        void rest_mesh(std::string val) { m_rest_mesh = strip_extension(val); }
        std::string init_mesh() const { return m_init_mesh; }
        void init_mesh(std::string val) { m_init_mesh = strip_extension(val); }
        std::string soln_mesh() const { return m_soln_mesh; }
        void soln_mesh(std::string val) { m_soln_mesh = strip_extension(val); m_soln_provided = true; }
        std::string handles() const { return m_handles; }
        void handles(std::string val) { m_handles = val; }
        int verbose() const { return m_verbose; }
        void verbose(int val) { m_verbose = val; }
        bool should_save_data() const { return m_should_save_data; }
        void should_save_data(bool val) { m_should_save_data = val; }
        bool soln_provided() const { return m_soln_provided; }

    private:
        /* "dir/bar.node" and "dir/bar" name the same .node/.ele pair */
        static std::string strip_extension(const std::string& raw) {
            const std::filesystem::path p(raw);
            const std::string parent = p.parent_path().string(), stem = p.stem().string();
            return parent.empty() ? stem : parent + "/" + stem;
        }
        std::string m_rest_mesh, m_init_mesh, m_soln_mesh, m_handles;
        int m_verbose = 1;
        bool m_should_save_data = true;
        bool m_soln_provided = false;
    };

    class GStep {
    public:
        enum class LineSearch { None, Backtracking };
        int max_iters() const { return m_max_iters; }
        void max_iters(int val) { m_max_iters = val; }
        LineSearch linesearch() const { return m_linesearch; }
        void linesearch(LineSearch val) { m_linesearch = val; }
        double kappa() const { return m_kappa; }
        void kappa(double val) { m_kappa = val; }

    private:
        int m_max_iters = 100;
        LineSearch m_linesearch = LineSearch::None;
        double m_kappa = 1.0;
    };

    enum class RotAwareness { ENABLED, DISABLED };
    enum class Reweighting { DISABLED, ENABLED };

    IO m_io;
    double m_tol = 1.e-11;
    int m_max_admm_iters = 5000;
    double m_reweighting_delay = 50;
    RotAwareness m_rot_awareness = RotAwareness::ENABLED;
    Reweighting m_reweighting = Reweighting::ENABLED;
    double m_gamma = 1.5;
    GStep m_gstep;
    ModelSettings m_model_settings;
    /* Extensions: the solver options the reference does not have, as in
     * wrapd_settings (lbfgs_m, rw_every, precision, prox_mode, leaf_size,
     * device, autotune); starts from wrapd_settings_default. */
    wrapd_settings m_gpu = defaults();

    bool parse_args(int argc, char** argv);
    void help() const;

    /* The flat C settings the library takes. */
    wrapd_settings to_c() const {
        wrapd_settings s = m_gpu;
        s.max_iters = m_max_admm_iters;
        s.tol = m_tol;
        s.rot_aware = m_rot_awareness == RotAwareness::ENABLED ? 1 : 0;
        s.reweighting = m_reweighting == Reweighting::ENABLED ? 1 : 0;
        s.rw_delay = static_cast<int>(m_reweighting_delay);
        s.gamma = m_gamma;
        s.global_iters = m_gstep.max_iters();
        s.global_ls = m_gstep.linesearch() == GStep::LineSearch::Backtracking ? 1 : 0;
        s.kappa = m_gstep.kappa();
        s.model = m_model_settings.elastic_model() == ModelSettings::ElasticModel::ARAP ? 1 : 0;
        s.youngs = m_model_settings.elastic_lame().youngs();
        s.poisson = m_model_settings.elastic_lame().poisson();
        s.beta_static = m_model_settings.elastic_beta_static();
        s.beta_min = m_model_settings.elastic_beta_min();
        s.beta_max = m_model_settings.elastic_beta_max();
        s.prox_iters = m_model_settings.elastic_prox_iters();
        s.verbose = m_io.verbose();
        return s;
    }

private:
    static wrapd_settings defaults() {
        wrapd_settings s;
        wrapd_settings_default(&s);
        return s;
    }
};

inline void Settings::help() const {
    std::cout << "\nArgs:\n"
                 " -rest, -init, -soln <mesh>   .node/.ele stems; -handles <file>: pinned vertex ids\n"
                 " -p <int> verbosity (1)   -s <0|1> save logs   -it <int> ADMM iterations (5000)\n"
                 " -tol <double> (1e-11)    -ra <0|1> rotation-aware (1)   -rw <0|1> reweighting (1)\n"
                 " -rw_delay <int> (50)     -gamma <double> (1.5)   -global_it <int> (100)\n"
                 " -global_ls <0|1> (0)     -kappa <double> (1)   -model <nh|arap>   -poisson <double> (0.45)\n"
                 " -beta_static (1), -beta_min (0.1), -beta_max (10)\n"
                 "Extensions: -youngs <double> (1e7)  -lbfgs_m <int> (6)  -rw_every <int>  -precision fp64|mixed\n"
                 "            -prox lbfgs|newton  -leaf <int>  -device <int>  -autotune 0|1\n\n";
}

inline bool Settings::parse_args(int argc, char** argv) {
    if (argc == 1) help();
    std::vector<std::string> cmds;
    std::vector<std::string> vals;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        const bool flag = a.size() > 1 && a[0] == '-' && !(a[1] >= '0' && a[1] <= '9') && a[1] != '.';
        if (flag) {
            cmds.push_back(a);
            vals.emplace_back();
        } else if (!vals.empty()) {
            vals.back() += a + " ";
        } else {
            throw std::runtime_error("Error: Unrecognized command-line argument: " + a);
        }
    }
    for (size_t i = 0; i < cmds.size(); ++i) {
        const std::string& a = cmds[i];
        std::istringstream v(vals[i]);
        auto geti = [&]() { int x = 0; v >> x; return x; };
        auto getd = [&]() { double x = 0; v >> x; return x; };
        auto gets = [&]() { std::string x; v >> x; return x; };
        if (a == "-help" || a == "--help" || a == "-h") { help(); return true; }
        else if (a == "-rest") m_io.rest_mesh(gets());
        else if (a == "-init") m_io.init_mesh(gets());
        else if (a == "-soln") m_io.soln_mesh(gets());
        else if (a == "-handles") m_io.handles(gets());
        else if (a == "-p") m_io.verbose(geti());
        else if (a == "-s") m_io.should_save_data(geti() != 0);
        else if (a == "-it") m_max_admm_iters = geti();
        else if (a == "-tol") m_tol = getd();
        else if (a == "-rotaware" || a == "-ra") {
            const int x = geti();
            if (x != 0 && x != 1) throw std::runtime_error("Error: Invalid value provided for argument -rotaware (or -ra)");
            m_rot_awareness = x ? RotAwareness::ENABLED : RotAwareness::DISABLED;
        } else if (a == "-reweighting" || a == "-rw") {
            const int x = geti();
            if (x != 0 && x != 1) throw std::runtime_error("Error: Invalid value provided for argument -reweighting (or -rw)");
            m_reweighting = x ? Reweighting::ENABLED : Reweighting::DISABLED;
        } else if (a == "-rw_delay") m_reweighting_delay = getd();
        else if (a == "-gamma") m_gamma = getd();
        else if (a == "-global_it") m_gstep.max_iters(geti());
        else if (a == "-global_ls") {
            const int x = geti();
            if (x != 0 && x != 1) throw std::runtime_error("Error: invalid value provided for argument -global_linesearch");
            m_gstep.linesearch(x ? GStep::LineSearch::Backtracking : GStep::LineSearch::None);
        } else if (a == "-kappa") m_gstep.kappa(getd());
        else if (a == "-model") m_model_settings.elastic_model(gets());
        else if (a == "-beta_static") m_model_settings.elastic_beta_static(getd());
        else if (a == "-beta_min") m_model_settings.elastic_beta_min(getd());
        else if (a == "-beta_max") m_model_settings.elastic_beta_max(getd());
        else if (a == "-poisson") m_model_settings.poisson(getd());
        else if (a == "-youngs") m_model_settings.youngs(getd());
        else if (a == "-lbfgs_m") m_gpu.lbfgs_m = geti();
        else if (a == "-rw_every") m_gpu.rw_every = geti();
        else if (a == "-precision") {
            const std::string p = gets();
            if (p != "fp64" && p != "mixed") throw std::runtime_error("Error: Invalid value provided for argument -precision");
            m_gpu.precision = p == "mixed" ? 1 : 0;
        } else if (a == "-prox") {
            const std::string p = gets();
            if (p != "lbfgs" && p != "newton") throw std::runtime_error("Error: Invalid value provided for argument -prox");
            m_gpu.prox_mode = p == "newton" ? 1 : 0;
        } else if (a == "-leaf") m_gpu.leaf_size = geti();
        else if (a == "-device") m_gpu.device = geti();
        else if (a == "-autotune") m_gpu.autotune = geti();
        else throw std::runtime_error("Error: Unrecognized command-line argument: " + a);
    }
    return false;
}

}  // namespace wrapd

#endif  // WRAPD_COMPAT_SETTINGS_HPP
