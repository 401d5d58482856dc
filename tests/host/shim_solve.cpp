// A solve through include/wrapd_gpu.hpp (wrapd::gpu::Solver), for the GPU
// test that compares it with the same solve through the Python mirror:
//
//   shim_solve <rest.bin> <init.bin> <tets.bin> <pins.bin> <youngs> <max_iters> <out_x.bin> <out_obj.bin>
//
// Inputs are raw float64 (n x 3) / int32 (m x 4, pins) files; writes the
// final positions (n x 3 float64) and the objectives log (float64).
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "wrapd_gpu.hpp"

namespace {

template <typename T>
std::vector<T> read_all(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f) / static_cast<long>(sizeof(T));
    std::fseek(f, 0, SEEK_SET);
    std::vector<T> v(n);
    const size_t got = n ? std::fread(v.data(), sizeof(T), n, f) : 0;
    std::fclose(f);
    if (got != static_cast<size_t>(n)) throw std::runtime_error(std::string("short read of ") + path);
    return v;
}

void write_all(const char* path, const std::vector<double>& v) {
    FILE* f = std::fopen(path, "wb");
    if (!f || std::fwrite(v.data(), sizeof(double), v.size(), f) != v.size())
        throw std::runtime_error(std::string("cannot write ") + path);
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: shim_solve rest init tets pins youngs max_iters out_x out_obj\n");
        return 2;
    }
    try {
        wrapd::gpu::Settings s;
        s.youngs = std::atof(argv[5]);
        s.max_iters = std::atoi(argv[6]);
        wrapd::gpu::Solver solver(s);
        const std::vector<int32_t> pins = read_all<int32_t>(argv[4]);
        solver.add_tetmesh(read_all<double>(argv[1]), read_all<double>(argv[2]), read_all<int32_t>(argv[3]));
        solver.set_pins(std::vector<int>(pins.begin(), pins.end()));
        solver.initialize(s);
        solver.solve();
        write_all(argv[7], solver.X());
        write_all(argv[8], solver.algorithm_data()->per_iter_objectives());
        std::printf("iterations %zu\n", solver.algorithm_data()->per_iter_objectives().size() - 1);
    } catch (const std::runtime_error& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
