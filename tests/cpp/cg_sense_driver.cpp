// Test driver for the C++ host interface (include/gadgetron_b200.hpp): reads
// raw little-endian arrays written by tests/test_cpp_host_gpu.py, runs the
// SENSE forward operator and a CG-SENSE solve through the C++ classes, and
// writes the results back as raw arrays.
//   argv: dir N mos W coils samples iterations
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "gadgetron_b200.hpp"

template <class T>
static std::vector<T> read_raw(const std::string &path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char *>(v.data()), n * sizeof(T));
    if (!f) throw std::runtime_error("cannot read " + path);
    return v;
}

template <class T>
static void write_raw(const std::string &path, const std::vector<T> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(T));
}

template <class T>
static T *to_device(const std::vector<T> &v) {
    T *p = nullptr;
    if (cudaMalloc(&p, v.size() * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}

int main(int argc, char **argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: %s dir N mos W coils samples iterations\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const uint64_t N = std::strtoull(argv[2], nullptr, 10), mos = std::strtoull(argv[3], nullptr, 10);
    const float W = std::strtof(argv[4], nullptr);
    const uint32_t C = (uint32_t)std::atoi(argv[5]);
    const uint64_t M = std::strtoull(argv[6], nullptr, 10);
    const uint32_t iters = (uint32_t)std::atoi(argv[7]);
    try {
        auto traj = read_raw<float>(dir + "/traj.f32", 2 * M);
        auto dcw = read_raw<float>(dir + "/sqrt_dcw.f32", M);
        auto csm = read_raw<float>(dir + "/csm.c64", 2 * C * N * N);
        auto img = read_raw<float>(dir + "/image.c64", 2 * N * N);
        auto data = read_raw<float>(dir + "/data.c64", 2 * C * M);
        float *d_traj = to_device(traj), *d_dcw = to_device(dcw), *d_csm = to_device(csm);
        float *d_img = to_device(img), *d_data = to_device(data);
        std::vector<float> y(2 * C * M), x(2 * N * N);
        float *d_y = to_device(y), *d_x = to_device(x);

        using namespace gadgetron_b200;
        const uint64_t n[2] = {N, N}, m[2] = {mos, mos};
        cuNonCartesianSenseOperator<2> E;
        E.setup(n, m, W);
        E.set_csm(d_csm, C);
        E.set_dcw(d_dcw);
        E.preprocess(d_traj, M);
        E.mult_M(d_img, d_y);
        cuCgSolver cg;
        cg.set_encoding_operator(E);
        cg.set_max_iterations(iters);
        cg.set_tc_tolerance(0.f);
        uint32_t its = cg.solve(d_data, d_x);
        cudaMemcpy(y.data(), d_y, y.size() * sizeof(float), cudaMemcpyDeviceToHost);
        cudaMemcpy(x.data(), d_x, x.size() * sizeof(float), cudaMemcpyDeviceToHost);
        write_raw(dir + "/y_cpp.c64", y);
        write_raw(dir + "/x_cpp.c64", x);
        std::printf("iterations %u\n", its);
        // errors are reported as exceptions, as in the reference
        try {
            cuNFFT_plan<2> bad(n, m, 1.0f);
            std::printf("no exception\n");
            return 1;
        } catch (const std::runtime_error &e) {
            std::printf("caught: %s\n", e.what());
        }
        for (void *p : {(void *)d_traj, (void *)d_dcw, (void *)d_csm, (void *)d_img, (void *)d_data, (void *)d_y,
                        (void *)d_x})
            cudaFree(p);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
