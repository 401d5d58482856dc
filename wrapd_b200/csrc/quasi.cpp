// quasi: the reference's command-line front end (samples/tests/quasi.cpp) on the
// B200 solver, through the C ABI of include/wrapd_gpu.h only.
//
//   quasi -rest <stem> -init <stem> -handles <file> [-soln <stem>] [flags]
//
// Flags and their parsing follow wrapd::Settings::parse_args
// (src/Settings.cpp:31-176): a token that starts with '-' and not with a digit
// or '.' opens a flag, the tokens after it are its value.  Inputs are TetGen
// .node/.ele pairs, 0- or 1-based (samples/utils/MeshIO.hpp:182-315), and a
// handles file of whitespace-separated vertex ids (quasi.cpp:146-159).
// Outputs, in the -out directory (the reference writes to its compile-time
// WRAPD_OUTPUT_DIR): objectives.txt, x_errors.txt, reweighted.txt and
// accumulated_time_s.txt as "<index> <value>" in %.14e (DataLog::write,
// samples/utils/DataLog.hpp:55-70), final_mesh.node/.ele
// (MeshIO.hpp:318-362) and final_mesh.obj with the boundary faces
// (TetMesh::need_faces, samples/utils/TetMesh.hpp:195-222; MeshIO.hpp:131-179).
//
// Extensions: -youngs E (the reference hard-codes 1e7 Pa, src/Lame.hpp:38),
// -out DIR, -lbfgs_m M, -rw_every N, -precision fp64|mixed,
// -prox lbfgs|newton|net (net: the prox network from -net FILE, a raw
// little-endian float32 blob), -leaf N, -device D, -autotune 0|1, -plan 1
// (print the host analysis and the factor's device pool sizes, then exit
// without touching the GPU).
#include <algorithm>
#include <array>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wrapd_gpu.h"

namespace {

struct Mesh {
    std::vector<double> xyz;    // n x 3
    std::vector<int32_t> tets;  // m x 4
};

[[noreturn]] void fail(const std::string& msg) { throw std::runtime_error(msg); }

// Mesh arguments lose their last extension (Settings::IO::strip_extension,
// src/Settings.hpp:81-91): "-rest bar.node" and "-rest bar" name the same pair.
std::string strip_extension(const std::string& raw) {
    const std::filesystem::path p(raw);
    const std::string parent = p.parent_path().string(), stem = p.stem().string();
    return parent.empty() ? stem : parent + "/" + stem;
}

// load_elenode: "<n> ..." header, then "<idx> a b c d" / "<idx> x y z" lines;
// indices start at 0 or 1 (decided by the first line).
Mesh load_elenode(const std::string& stem) {
    Mesh m;
    {
        std::ifstream f(stem + ".ele");
        if (!f) fail("**TetMesh Error: Could not load " + stem + ".ele");
        std::string line;
        std::getline(f, line);
        int n = 0;
        std::istringstream(line) >> n;
        m.tets.assign(4 * (size_t)std::max(n, 0), -1);
        std::vector<char> seen(std::max(n, 0), 0);
        bool one_based = false;
        for (int i = 0; i < n; ++i) {
            if (!std::getline(f, line)) fail("**TetMesh Error: Your indices are bad for file " + stem + ".ele");
            std::istringstream ls(line);
            long idx;
            int v[4];
            ls >> idx >> v[0] >> v[1] >> v[2] >> v[3];
            if (i == 0 && idx == 1) one_based = true;
            if (one_based) { idx -= 1; for (int& x : v) x -= 1; }
            if (idx < 0 || idx >= n) fail("**TetMesh Error: Your indices are bad for file " + stem + ".ele");
            for (int k = 0; k < 4; ++k) m.tets[4 * idx + k] = v[k];
            seen[idx] = 1;
        }
        for (char c : seen) if (!c) fail("**TetMesh Error: Your indices are bad for file " + stem + ".ele");
    }
    {
        std::ifstream f(stem + ".node");
        if (!f) fail("**TetMesh Error: Could not load " + stem + ".node");
        std::string line;
        std::getline(f, line);
        int n = 0;
        std::istringstream(line) >> n;
        m.xyz.assign(3 * (size_t)std::max(n, 0), 0.0);
        std::vector<char> seen(std::max(n, 0), 0);
        bool one_based = false;
        for (int i = 0; i < n; ++i) {
            if (!std::getline(f, line)) fail("**TetMesh Error: Your indices are bad for file " + stem + ".node");
            std::istringstream ls(line);
            long idx;
            double x, y, z;
            ls >> idx >> x >> y >> z;
            if (i == 0 && idx == 1) one_based = true;
            if (one_based) idx -= 1;
            if (idx < 0 || idx >= n) fail("**TetMesh Error: Your indices are bad for file " + stem + ".node");
            m.xyz[3 * idx] = x; m.xyz[3 * idx + 1] = y; m.xyz[3 * idx + 2] = z;
            seen[idx] = 1;
        }
        for (char c : seen) if (!c) fail("**TetMesh Error: Your indices are bad for file " + stem + ".node");
    }
    if (m.xyz.empty() || m.tets.empty()) fail("**TetMesh Error: Problem loading files");
    return m;
}

std::vector<int32_t> load_handles(const std::string& path) {
    std::vector<int32_t> pins;
    std::ifstream f(path);
    long v;
    while (f >> v) pins.push_back(static_cast<int32_t>(v));
    return pins;
}

void write_log(const std::string& path, const std::vector<double>& v) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) fail("Error: Unable to open file.");
    for (size_t i = 0; i < v.size(); ++i) std::fprintf(f, "%.14e %.14e\n", double(i), v[i]);
    std::fclose(f);
}

void save_elenode(const std::string& stem, const std::vector<double>& X, const std::vector<int32_t>& tets) {
    FILE* f = std::fopen((stem + ".ele").c_str(), "w");
    if (!f) fail("Error: Unable to open file.");
    const size_t m = tets.size() / 4, n = X.size() / 3;
    std::fprintf(f, "%zu 4 0\n", m);
    for (size_t i = 0; i < m; ++i)
        std::fprintf(f, "\t%zu %d %d %d %d\n", i, tets[4 * i], tets[4 * i + 1], tets[4 * i + 2], tets[4 * i + 3]);
    std::fprintf(f, "# Generated by mclscene (www.mattoverby.net)");
    std::fclose(f);
    f = std::fopen((stem + ".node").c_str(), "w");
    if (!f) fail("Error: Unable to open file.");
    std::fprintf(f, "%zu 3 0 0\n", n);
    for (size_t i = 0; i < n; ++i) std::fprintf(f, "\t%zu %.15e %.15e %.15e\n", i, X[3 * i], X[3 * i + 1], X[3 * i + 2]);
    std::fprintf(f, "# Generated by mclscene (www.mattoverby.net)");
    std::fclose(f);
}

// Boundary faces: faces used by exactly one tet, keyed by their sorted vertex
// ids, written with the vertex order of that tet's face (p0 p1 p3, p0 p2 p1,
// p0 p3 p2, p1 p2 p3).  Emitted in order of first appearance (the reference
// emits them in hash-table order; the set of oriented faces is the same).
void save_obj(const std::string& path, const std::vector<double>& X, const std::vector<int32_t>& tets) {
    std::map<std::array<int, 3>, std::pair<int, size_t>> count;   // sorted key -> (uses, first index)
    std::vector<std::array<int, 3>> faces;
    const size_t m = tets.size() / 4;
    for (size_t t = 0; t < m; ++t) {
        const int p0 = tets[4 * t], p1 = tets[4 * t + 1], p2 = tets[4 * t + 2], p3 = tets[4 * t + 3];
        const std::array<int, 3> fs[4] = {{p0, p1, p3}, {p0, p2, p1}, {p0, p3, p2}, {p1, p2, p3}};
        for (const auto& fc : fs) {
            std::array<int, 3> key = fc;
            std::sort(key.begin(), key.end());
            auto it = count.find(key);
            if (it == count.end()) {
                count.emplace(key, std::make_pair(1, faces.size()));
                faces.push_back(fc);
            } else {
                it->second.first += 1;
            }
        }
    }
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) fail("Error: Unable to open file.");
    std::fprintf(f, "# Generated with mclscene by Matt Overby (www.mattoverby.net)");
    const size_t n = X.size() / 3;
    for (size_t i = 0; i < n; ++i) std::fprintf(f, "\nv %.15e %.15e %.15e", X[3 * i], X[3 * i + 1], X[3 * i + 2]);
    std::vector<char> boundary(faces.size(), 0);
    for (const auto& kv : count)
        if (kv.second.first == 1) boundary[kv.second.second] = 1;
    for (size_t i = 0; i < faces.size(); ++i)
        if (boundary[i]) std::fprintf(f, "\nf %d %d %d", faces[i][0] + 1, faces[i][1] + 1, faces[i][2] + 1);
    std::fprintf(f, "\n");
    std::fclose(f);
}

void help() {
    std::printf(
        "\nArgs (as the reference's quasi):\n"
        " -rest, -init, -soln <stem>   .node/.ele meshes; -handles <file>: pinned vertex ids\n"
        " -it N (5000)  -tol T (1e-11)  -ra 0|1 (1)  -rw 0|1 (1)  -rw_delay N (50)  -gamma G (1.5)\n"
        " -global_it N (100)  -global_ls 0|1  -kappa K (1)  -model nh|arap  -poisson P (0.45)\n"
        " -beta_static B (1)  -beta_min B (0.1)  -beta_max B (10)  -p 0|1  -s 0|1 (1)\n"
        "Extensions: -youngs E (1e7)  -out DIR (.)  -lbfgs_m M (6)  -rw_every N  -precision fp64|mixed\n"
        "            -prox lbfgs|newton|net  -net FILE  -leaf N  -device D  -autotune 0|1\n"
        "            -plan 1 (print the analysis and device pool sizes, no GPU, then exit)\n\n");
}

int run(int argc, char** argv) {
    if (argc == 1) { help(); return 0; }
    std::vector<std::string> cmds;
    std::vector<std::string> vals;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        const bool flag = a.size() > 1 && a[0] == '-' && !(a[1] >= '0' && a[1] <= '9') && a[1] != '.';
        if (flag) { cmds.push_back(a); vals.emplace_back(); }
        else if (!vals.empty()) vals.back() += a + " ";
        else fail("Error: Unrecognized command-line argument: " + a);
    }
    wrapd_settings s;
    wrapd_settings_default(&s);
    std::string rest, init, soln, handles, out = ".", net;
    int save = 1, plan_only = 0;
    for (size_t i = 0; i < cmds.size(); ++i) {
        const std::string& a = cmds[i];
        std::istringstream v(vals[i]);
        auto geti = [&]() { long x = 0; v >> x; return static_cast<int>(x); };
        auto getd = [&]() { double x = 0; v >> x; return x; };
        auto gets = [&]() { std::string x; v >> x; return x; };
        if (a == "-help" || a == "--help" || a == "-h") { help(); return 0; }
        else if (a == "-rest") rest = strip_extension(gets());
        else if (a == "-init") init = strip_extension(gets());
        else if (a == "-soln") soln = strip_extension(gets());
        else if (a == "-handles") handles = gets();
        else if (a == "-p") s.verbose = geti();
        else if (a == "-s") save = geti();
        else if (a == "-it") s.max_iters = geti();
        else if (a == "-tol") s.tol = getd();
        else if (a == "-rotaware" || a == "-ra") {
            s.rot_aware = geti();
            if (s.rot_aware != 0 && s.rot_aware != 1) fail("Error: Invalid value provided for argument -rotaware (or -ra)");
        } else if (a == "-reweighting" || a == "-rw") {
            s.reweighting = geti();
            if (s.reweighting != 0 && s.reweighting != 1) fail("Error: Invalid value provided for argument -reweighting (or -rw)");
        } else if (a == "-rw_delay") s.rw_delay = geti();
        else if (a == "-gamma") s.gamma = getd();
        else if (a == "-global_it") s.global_iters = geti();
        else if (a == "-global_ls") {
            s.global_ls = geti();
            if (s.global_ls != 0 && s.global_ls != 1) fail("Error: invalid value provided for argument -global_linesearch");
        } else if (a == "-kappa") s.kappa = getd();
        else if (a == "-model") {
            const std::string m = gets();
            if (m == "arap") s.model = 1;
            else if (m == "nh") s.model = 0;
            else fail("Error: Invalid elastic model: " + m);
        } else if (a == "-beta_static") s.beta_static = getd();
        else if (a == "-beta_min") s.beta_min = getd();
        else if (a == "-beta_max") s.beta_max = getd();
        else if (a == "-poisson") s.poisson = getd();
        else if (a == "-youngs") s.youngs = getd();
        else if (a == "-out") out = gets();
        else if (a == "-lbfgs_m") s.lbfgs_m = geti();
        else if (a == "-rw_every") s.rw_every = geti();
        else if (a == "-precision") {
            const std::string p = gets();
            if (p == "fp64") s.precision = 0;
            else if (p == "mixed") s.precision = 1;
            else fail("Error: Invalid value provided for argument -precision");
        } else if (a == "-prox") {
            const std::string p = gets();
            if (p == "lbfgs") s.prox_mode = 0;
            else if (p == "newton") s.prox_mode = 1;
            else if (p == "net") s.prox_mode = 2;
            else fail("Error: Invalid value provided for argument -prox");
        } else if (a == "-net") net = gets();
        else if (a == "-leaf") s.leaf_size = geti();
        else if (a == "-device") s.device = geti();
        else if (a == "-autotune") s.autotune = geti();
        else if (a == "-plan") plan_only = geti();
        else fail("Error: Unrecognized command-line argument: " + a);
    }
    const std::vector<int32_t> pins = load_handles(handles);
    const Mesh R = load_elenode(rest), I = load_elenode(init);
    if (R.xyz.size() != I.xyz.size())
        fail("Error: Rest mesh and init mesh do not have the same number of vertices.");
    Mesh S;
    if (!soln.empty()) S = load_elenode(soln);
    const int nv = static_cast<int>(R.xyz.size() / 3), nt = static_cast<int>(R.tets.size() / 4);

    if (plan_only) {
        wrapd_plan* p = nullptr;
        if (wrapd_plan_create(R.xyz.data(), nv, R.tets.data(), nt, pins.data(), static_cast<int>(pins.size()),
                              s.leaf_size, &p) != WRAPD_OK)
            fail(wrapd_last_error(nullptr));
        int64_t info[8];
        wrapd_plan_info(p, info);
        wrapd_plan_destroy(p);
        std::printf("free vertices %lld\nfronts %lld\nlevels %lld\nfactor entries %lld\n"
                    "factor flops %lld\nF pool bytes %lld\nY pool bytes %lld\n",
                    (long long)info[0], (long long)info[1], (long long)info[2], (long long)info[3],
                    (long long)info[7], (long long)info[4], (long long)info[5]);
        return 0;
    }
    wrapd_handle* h = nullptr;
    if (wrapd_create(&s, &h) != WRAPD_OK) fail(wrapd_last_error(nullptr));
    auto check = [&](int rc) {
        if (rc != WRAPD_OK) {
            const std::string m = wrapd_last_error(h);
            wrapd_destroy(h);
            fail(m);
        }
    };
    check(wrapd_add_tetmesh(h, R.xyz.data(), I.xyz.data(), soln.empty() ? nullptr : S.xyz.data(), nv, R.tets.data(),
                            nt, pins.data(), static_cast<int>(pins.size())));
    if (s.prox_mode == 2) {
        std::vector<float> blob(WRAPD_NET_BLOB);
        FILE* f = net.empty() ? nullptr : std::fopen(net.c_str(), "rb");
        if (!f || std::fread(blob.data(), sizeof(float), blob.size(), f) != blob.size()) {
            if (f) std::fclose(f);
            wrapd_destroy(h);
            fail("Error: -prox net needs -net FILE with " + std::to_string(WRAPD_NET_BLOB) + " float32 values");
        }
        std::fclose(f);
        check(wrapd_set_prox_net(h, blob.data(), WRAPD_NET_BLOB));
    }
    check(wrapd_initialize(h));
    std::vector<double> X(3 * (size_t)nv);
    check(wrapd_solve(h, X.data()));
    auto get_log = [&](int which) {
        int n = 0;
        check(wrapd_get_log(h, which, nullptr, 0, &n));
        std::vector<double> v(n);
        if (n) check(wrapd_get_log(h, which, v.data(), n, &n));
        return v;
    };
    double rt[6] = {0, 0, 0, 0, 0, 0};
    check(wrapd_get_runtime(h, rt));
    if (save) {
        write_log(out + "/objectives.txt", get_log(WRAPD_LOG_OBJECTIVES));
        write_log(out + "/x_errors.txt", get_log(WRAPD_LOG_X_ERRORS));
        write_log(out + "/reweighted.txt", get_log(WRAPD_LOG_REWEIGHTED));
        write_log(out + "/accumulated_time_s.txt", get_log(WRAPD_LOG_ACCUMULATED_TIME_S));
    }
    save_elenode(out + "/final_mesh", X, I.tets);
    save_obj(out + "/final_mesh.obj", X, I.tets);
    if (s.verbose > 0) {
        const double l = rt[1] / 1000.0, g = rt[2] / 1000.0, r = rt[3] / 1000.0;
        std::printf("Final accumulated time (s): %f\n-- Local step (s): %f\n-- Global step (s): %f\n"
                    "-- Refactor step (s): %f\n", l + g + r, l, g, r);
    }
    wrapd_destroy(h);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
}
