/* ModelSettings.hpp -- wrapd::ModelSettings (the reference's
 * src/ModelSettings.hpp:30-95): elastic model, Lame parameters and the
 * reweighting bounds, with the reference's defaults (NH, nu = 0.45 at
 * 1e7 Pa, beta 1 / 0.1 / 10, 20 prox iterations).  Extension: youngs(E) sets
 * Young's modulus (the reference fixes it at 1e7 Pa); poisson(v) keeps it. */
#ifndef WRAPD_COMPAT_MODELSETTINGS_HPP
#define WRAPD_COMPAT_MODELSETTINGS_HPP

#include <stdexcept>
#include <string>

#include "Lame.hpp"
#include "Math.hpp"

namespace wrapd {

class ModelSettings {
public:
    enum class ElasticModel { ARAP, NH };
    enum class ProxLSMethod { None, MoreThuente, Backtracking, BacktrackingCubic, WeakWolfeBisection };

    ModelSettings() : m_elastic_lame(Lame::preset(0.45)) {}

    ElasticModel elastic_model() const { return m_elastic_model; }
    void elastic_model(std::string val) {
        if (val == "arap") m_elastic_model = ElasticModel::ARAP;
        else if (val == "nh") m_elastic_model = ElasticModel::NH;
        else throw std::runtime_error("Error: Invalid input for -elastic_model");
    }
    void poisson(double val) { m_poisson = val; m_elastic_lame = Lame(m_youngs, val); }
    void youngs(double val) { m_youngs = val; m_elastic_lame = Lame(val, m_poisson); }
    const Lame& elastic_lame() const { return m_elastic_lame; }
    void elastic_lame(const Lame& val) { m_elastic_lame = val; }

    double elastic_beta_static() const { return m_elastic_beta_static; }
    void elastic_beta_static(double val) { m_elastic_beta_static = val; }
    double elastic_beta_min() const { return m_elastic_beta_min; }
    void elastic_beta_min(double val) { m_elastic_beta_min = val; }
    double elastic_beta_max() const { return m_elastic_beta_max; }
    void elastic_beta_max(double val) { m_elastic_beta_max = val; }
    ProxLSMethod elastic_prox_ls_method() const { return ProxLSMethod::BacktrackingCubic; }
    int elastic_prox_iters() const { return m_elastic_prox_iters; }

private:
    ElasticModel m_elastic_model = ElasticModel::NH;
    double m_youngs = 1.0e7, m_poisson = 0.45;
    Lame m_elastic_lame;
    double m_elastic_beta_static = 1.0, m_elastic_beta_min = 0.1, m_elastic_beta_max = 10.0;
    int m_elastic_prox_iters = 20;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_MODELSETTINGS_HPP
