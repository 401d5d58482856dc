// Test infrastructure: a driver for the reference's own solver, compiled
// straight from the reference sources (see oracle/Makefile).  It is the
// reference's `quasi` flow (samples/tests/quasi.cpp:44-144) with three
// differences that need no change to the reference's files:
//   * Young's modulus comes from `-youngs E` (the reference hard-codes
//     1e7 Pa at src/Lame.hpp:38); the Lame object inside Settings is replaced
//     through its public constructor and setters before the Solver copies it.
//   * outputs go to `-out DIR` instead of the compiled-in WRAPD_OUTPUT_DIR;
//   * besides the reference's logs it writes the inner L-BFGS iteration
//     counts, the local/global delta-AL columns, the run times and the final
//     positions as raw little-endian doubles (final_x.bin, n x 3 row-major);
//   * the final mesh files (final_mesh.node/.ele/.obj) are written with the
//     reference's own MeshIO calls, as quasi.cpp:113-130 does;
//   * built as quasi_ref_m5 (WRAPD_REF_PATCHED, the patched copy described in
//     oracle/Makefile: global L-BFGS history 5), it also takes `-rw_every N`,
//     which sets the reweight-every-N hook of the patched System.cpp.
// Every other flag is handed to wrapd::Settings::parse_args unchanged.
//
// Only tests, the CPU baseline of bench.py and fixture generation run it.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "AddMeshes.hpp"
#include "MeshIO.hpp"

namespace {

std::vector<int> load_handles(const std::string& path) {
    std::vector<int> pins;
    std::ifstream in(path.c_str());
    if (!in.is_open()) throw std::runtime_error("cannot open handles file " + path);
    std::string line;
    while (std::getline(in, line)) {
        std::stringstream ss(line);
        int idx;
        while (ss >> idx) pins.push_back(idx);
    }
    return pins;
}

template <typename T>
void write_log(const std::string& path, const std::vector<T>& v) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    for (size_t i = 0; i < v.size(); ++i)
        std::fprintf(f, "%.14e %.14e\n", static_cast<double>(i), static_cast<double>(v[i]));
    std::fclose(f);
}

}  // namespace

#ifdef WRAPD_REF_PATCHED
// Read by the patched System::possibly_update_weights (0: the gamma rule).
int wrapd_ref_rw_every = 0;
#endif

int main(int argc, char** argv) {
    double youngs = 1.0e7;
    double poisson = 0.45;
    std::string outdir = ".";
    std::vector<char*> pass;
    pass.push_back(argv[0]);
    for (int i = 1; i < argc; ++i) {
        std::string a(argv[i]);
        if (a == "-youngs" && i + 1 < argc) { youngs = std::atof(argv[++i]); continue; }
        if (a == "-out" && i + 1 < argc) { outdir = argv[++i]; continue; }
        if (a == "-rw_every" && i + 1 < argc) {
#ifdef WRAPD_REF_PATCHED
            wrapd_ref_rw_every = std::atoi(argv[++i]);
            continue;
#else
            std::fprintf(stderr, "-rw_every needs the patched build (quasi_ref_m5)\n");
            return EXIT_FAILURE;
#endif
        }
        if (a == "-poisson" && i + 1 < argc) poisson = std::atof(argv[i + 1]);
        pass.push_back(argv[i]);
    }

    wrapd::Settings settings;
    settings.m_io.should_save_data(true);
    settings.parse_args(static_cast<int>(pass.size()), pass.data());
    // Replace the hard-coded 1e7 Pa material with (youngs, poisson).
    const_cast<wrapd::Lame&>(settings.m_model_settings.elastic_lame()) = wrapd::Lame(youngs, poisson);

    std::vector<int> pins = load_handles(settings.m_io.handles());
    auto solver = std::make_shared<wrapd::Solver>(settings);

    auto rest_mesh = mcl::TetMesh::create();
    auto init_mesh = mcl::TetMesh::create();
    mcl::meshio::load_elenode(rest_mesh.get(), settings.m_io.rest_mesh());
    mcl::meshio::load_elenode(init_mesh.get(), settings.m_io.init_mesh());
    std::shared_ptr<mcl::TetMesh> soln_mesh;
    if (!settings.m_io.soln_mesh().empty()) {
        soln_mesh = mcl::TetMesh::create();
        mcl::meshio::load_elenode(soln_mesh.get(), settings.m_io.soln_mesh());
    } else {
        soln_mesh = rest_mesh;
    }
    rest_mesh->flags |= (settings.m_model_settings.elastic_model() == wrapd::ModelSettings::ElasticModel::ARAP)
                            ? binding::ARAP : binding::NH;
    init_mesh->flags = rest_mesh->flags;
    binding::add_tetmesh(solver.get(), rest_mesh, init_mesh, soln_mesh, pins, settings);

    solver->initialize(settings);
    solver->solve();

    wrapd::AlgorithmData* ad = solver->algorithm_data();
    write_log(outdir + "/objectives.txt", ad->per_iter_objectives());
    write_log(outdir + "/x_errors.txt", ad->per_iter_state_x_errors());
    write_log(outdir + "/reweighted.txt", ad->per_iter_reweighted());
    write_log(outdir + "/accumulated_time_s.txt", ad->per_iter_accumulated_time_s());
    // The reference stores inner iteration counts with operator[] into reserved
    // capacity (src/GlobalStepBehavior.hpp:254) without growing the vector, so
    // its size() stays 0; read the m_iter entries from the buffer directly.
    {
        const int* it = ad->per_iter_inner_iters().data();
        std::vector<int> inner(it, it + ad->m_iter);
        write_log(outdir + "/inner_iters.txt", inner);
    }
    write_log(outdir + "/ls_delta_al.txt", ad->m_per_iter_ls_delta_auglag);
    write_log(outdir + "/gs_delta_al.txt", ad->m_per_iter_gs_delta_auglag);
    {
        FILE* f = std::fopen((outdir + "/runtime.txt").c_str(), "w");
        const wrapd::RuntimeData& r = ad->m_runtime;
        std::fprintf(f, "setup_ms %.6f\nlocal_ms %.6f\nglobal_ms %.6f\nrefactor_ms %.6f\nfinish_ms %.6f\n"
                        "inner_iters %d\niters %d\n",
                     r.setup_solve_ms, r.local_ms, r.global_ms, r.refactor_ms, r.finish_solve_ms,
                     r.inner_iters, ad->m_iter);
        std::fclose(f);
    }
    {
        const wrapd::math::MatX3& X = solver->m_system->X();
        std::vector<double> rowmajor(static_cast<size_t>(X.rows()) * 3);
        for (int i = 0; i < X.rows(); ++i)
            for (int c = 0; c < 3; ++c) rowmajor[static_cast<size_t>(i) * 3 + c] = X(i, c);
        FILE* f = std::fopen((outdir + "/final_x.bin").c_str(), "wb");
        std::fwrite(rowmajor.data(), sizeof(double), rowmajor.size(), f);
        std::fclose(f);
    }
    {
        auto final_mesh = mcl::TetMesh::create();
        final_mesh->tets = init_mesh->tets;
        const wrapd::math::MatX3& X = solver->m_system->X();
        final_mesh->vertices.resize(init_mesh->vertices.size());
        for (int i = 0; i < static_cast<int>(final_mesh->vertices.size()); i++) final_mesh->vertices[i] = X.row(i);
        mcl::meshio::save_elenode(final_mesh.get(), outdir + "/final_mesh");
        final_mesh->need_faces(true);
        auto obj = mcl::TriangleMesh::create();
        obj->vertices = final_mesh->vertices;
        obj->faces = final_mesh->faces;
        mcl::meshio::save_obj(obj.get(), outdir + "/final_mesh.obj");
    }
    return EXIT_SUCCESS;
}
