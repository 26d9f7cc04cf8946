// Test infrastructure, not product code: a C-ABI driver over the reference's
// own GPU reconstruction path (cuNFFT_impl<float,D,STANDARD>,
// cuNonCartesianSenseOperator, cuCgSolver), built from the reference's
// sources by oracle/build_ref.py into oracle/_ref/libgbref.so.  Only the
// tests, smoke() and the bench's reference legs load it, to compare the
// product's outputs with the reference's on the same seeded inputs.
//
// Every entry takes HOST buffers in the reference's x-fastest layouts, copies
// them into cuNDArrays, runs the reference API exactly as its callers do, and
// copies the result back.  Errors (C++ exceptions of the reference, CUDA
// errors) become a nonzero return and a message in gbref_last_error().
//
// Layouts (x fastest, as the reference's cuNDArray dims list them):
//   trajectory  [M, F] of vector_td<float,D>       (nfft/NFFT.h:67-68)
//   image       [N_0..N_{D-1}, F, B] complext<float> (or the oversampled size)
//   samples     [M, F, B] complext<float>
//   dcw         [M, F] float
//   csm         [N_0..N_{D-1}, C] complext<float>   (senseOperator.h:26-35)
//   SENSE data  [M*F, C] (gadgets/pmri/gpuCgSenseGadget.cpp:155-161)
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cuNFFT.h"
#include "cuNDArray.h"
#include "cuNDArray_blas.h"
#include "cuNDArray_elemwise.h"
#include "cuNDArray_operators.h"
#include "cuCgSolver.h"
#include "cuNonCartesianSenseOperator.h"

using namespace Gadgetron;

namespace {

thread_local std::string g_err;

void cuda_ok(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T> cuNDArray<T> upload(const std::vector<size_t> &dims, const void *host) {
    cuNDArray<T> a(dims);
    cuda_ok(cudaMemcpy(a.get_data_ptr(), host, a.get_number_of_elements() * sizeof(T), cudaMemcpyHostToDevice),
            "upload");
    return a;
}

template <class T> void download(const cuNDArray<T> &a, void *host) {
    cuda_ok(cudaMemcpy(host, a.get_data_ptr(), a.get_number_of_elements() * sizeof(T), cudaMemcpyDeviceToHost),
            "download");
}

template <unsigned D> vector_td<size_t, D> vec(const uint64_t *v) {
    vector_td<size_t, D> r;
    for (unsigned d = 0; d < D; d++) r[d] = (size_t)v[d];
    return r;
}

template <unsigned D> std::vector<size_t> dims_of(const uint64_t *v) {
    std::vector<size_t> r;
    for (unsigned d = 0; d < D; d++) r.push_back((size_t)v[d]);
    return r;
}

NFFT_comp_mode comp_mode(int m) {
    switch (m) {
    case 0: return NFFT_comp_mode::FORWARDS_C2NC;
    case 1: return NFFT_comp_mode::FORWARDS_NC2C;
    case 2: return NFFT_comp_mode::BACKWARDS_C2NC;
    case 3: return NFFT_comp_mode::BACKWARDS_NC2C;
    }
    throw std::runtime_error("unknown compute mode");
}

template <unsigned D>
cuNDArray<vector_td<float, D>> upload_traj(const float *traj, uint64_t M, uint64_t F) {
    return upload<vector_td<float, D>>({(size_t)M, (size_t)F}, traj);
}

// image dims [N..., F, B] (or oversampled); samples [M, F, B]
template <unsigned D>
int nfft_compute(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
                 const void *in, void *out, const float *dcw, int mode, uint64_t B, int oversampled_image,
                 int conv_type) {
    auto plan = NFFT<cuNDArray, float, D>::make_plan(vec<D>(n), vec<D>(mos), W, (ConvolutionType)conv_type);
    auto t = upload_traj<D>(traj, M, F);
    plan->preprocess(t, NFFT_prep_mode::ALL);
    std::vector<size_t> img = dims_of<D>(oversampled_image ? mos : n);
    img.push_back((size_t)F);
    img.push_back((size_t)B);
    std::vector<size_t> smp = {(size_t)M, (size_t)F, (size_t)B};
    const NFFT_comp_mode cm = comp_mode(mode);
    const bool c2nc = cm == NFFT_comp_mode::FORWARDS_C2NC || cm == NFFT_comp_mode::BACKWARDS_C2NC;
    auto a_in = upload<complext<float>>(c2nc ? img : smp, in);
    cuNDArray<complext<float>> a_out(c2nc ? smp : img);
    cuNDArray<float> a_dcw;
    if (dcw) a_dcw = upload<float>({(size_t)M, (size_t)F}, dcw);
    plan->compute(a_in, a_out, dcw ? &a_dcw : nullptr, cm);
    cuda_ok(cudaDeviceSynchronize(), "compute");
    download(a_out, out);
    return 0;
}

template <unsigned D>
int nfft_mult_MH_M(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
                   const void *in, void *out, const float *dcw, uint64_t B) {
    auto plan = NFFT<cuNDArray, float, D>::make_plan(vec<D>(n), vec<D>(mos), W, ConvolutionType::STANDARD);
    auto t = upload_traj<D>(traj, M, F);
    plan->preprocess(t, NFFT_prep_mode::ALL);
    std::vector<size_t> img = dims_of<D>(n);
    img.push_back((size_t)F);
    img.push_back((size_t)B);
    auto a_in = upload<complext<float>>(img, in);
    cuNDArray<complext<float>> a_out(img);
    cuNDArray<float> a_dcw;
    if (dcw) a_dcw = upload<float>({(size_t)M, (size_t)F}, dcw);
    plan->mult_MH_M(a_in, a_out, dcw ? &a_dcw : nullptr);
    cuda_ok(cudaDeviceSynchronize(), "mult_MH_M");
    download(a_out, out);
    return 0;
}

// standalone convolution: conv 0 = C2NC (os grid -> samples), 1 = NC2C
template <unsigned D>
int nfft_convolve(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
                  const void *in, void *out, int conv, uint64_t B, int accumulate) {
    auto plan = NFFT<cuNDArray, float, D>::make_plan(vec<D>(n), vec<D>(mos), W, ConvolutionType::STANDARD);
    auto t = upload_traj<D>(traj, M, F);
    plan->preprocess(t, NFFT_prep_mode::ALL);
    std::vector<size_t> grid = dims_of<D>(mos);
    grid.push_back((size_t)F);
    grid.push_back((size_t)B);
    std::vector<size_t> smp = {(size_t)M, (size_t)F, (size_t)B};
    auto a_in = upload<complext<float>>(conv == 0 ? grid : smp, in);
    // accumulate adds onto the caller's output: upload it
    auto a_out = upload<complext<float>>(conv == 0 ? smp : grid, out);
    plan->convolve(a_in, a_out, conv == 0 ? NFFT_conv_mode::C2NC : NFFT_conv_mode::NC2C, accumulate != 0);
    cuda_ok(cudaDeviceSynchronize(), "convolve");
    download(a_out, out);
    return 0;
}

// fft (dir 0 forwards, 1 backwards) or deapodize (dir 2 image domain, 3
// Fourier domain) in place on an oversampled array [mos..., F*B]
template <unsigned D>
int nfft_fft_deapod(const uint64_t *n, const uint64_t *mos, float W, void *data, uint64_t FB, int op,
                    int do_scale) {
    auto plan = NFFT<cuNDArray, float, D>::make_plan(vec<D>(n), vec<D>(mos), W, ConvolutionType::STANDARD);
    std::vector<size_t> grid = dims_of<D>(mos);
    grid.push_back((size_t)FB);
    auto a = upload<complext<float>>(grid, data);
    if (op == 0 || op == 1)
        plan->fft(a, op == 0 ? NFFT_fft_mode::FORWARDS : NFFT_fft_mode::BACKWARDS, do_scale != 0);
    else
        plan->deapodize(a, op == 3);
    cuda_ok(cudaDeviceSynchronize(), "fft/deapodize");
    download(a, data);
    return 0;
}

template <unsigned D>
boost::shared_ptr<cuNonCartesianSenseOperator<float, D>>
make_sense(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
           const void *csm, uint64_t C, const float *dcw) {
    auto E = boost::make_shared<cuNonCartesianSenseOperator<float, D>>(ConvolutionType::STANDARD);
    std::vector<size_t> dom = dims_of<D>(n);
    dom.push_back((size_t)F);
    E->set_domain_dimensions(dom);
    E->set_codomain_dimensions({(size_t)(M * F), (size_t)C});
    if (dcw) E->set_dcw(boost::make_shared<cuNDArray<float>>(upload<float>({(size_t)M, (size_t)F}, dcw)));
    std::vector<size_t> cd = dims_of<D>(n);
    cd.push_back((size_t)C);
    E->set_csm(boost::make_shared<cuNDArray<complext<float>>>(upload<complext<float>>(cd, csm)));
    E->setup(vec<D>(n), vec<D>(mos), W);
    auto t = upload_traj<D>(traj, M, F);
    E->preprocess(&t);
    return E;
}

template <unsigned D>
int sense_mult(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
               const void *csm, uint64_t C, const float *dcw, const void *in, void *out, int adjoint) {
    auto E = make_sense<D>(n, mos, W, traj, M, F, csm, C, dcw);
    std::vector<size_t> dom = dims_of<D>(n);
    dom.push_back((size_t)F);
    std::vector<size_t> cod = {(size_t)(M * F), (size_t)C};
    auto a_in = upload<complext<float>>(adjoint ? cod : dom, in);
    cuNDArray<complext<float>> a_out(adjoint ? dom : cod);
    if (adjoint)
        E->mult_MH(&a_in, &a_out, false);
    else
        E->mult_M(&a_in, &a_out, false);
    cuda_ok(cudaDeviceSynchronize(), "sense");
    download(a_out, out);
    return 0;
}

// cuCgSolver that copies every iterate to a host buffer (solver_dump is the
// reference's per-iteration hook, cgSolver.h:98,152)
template <class T> class RecordingCg : public cuCgSolver<T> {
  public:
    RecordingCg(char *dst, size_t bytes) : dst_(dst), bytes_(bytes) {}
    void solver_dump(cuNDArray<T> *x) override {
        if (!dst_) return;
        cuda_ok(cudaMemcpy(dst_ + k_ * bytes_, x->get_data_ptr(), bytes_, cudaMemcpyDeviceToHost), "dump");
        k_++;
    }
    int k_ = 0;

  private:
    char *dst_;
    size_t bytes_;
};

template <unsigned D>
int cg_sense(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
             const void *csm, uint64_t C, const float *dcw, const void *data, void *x_out, int iterations,
             float tc_tolerance, void *iterates, int *iterations_run) {
    auto E = make_sense<D>(n, mos, W, traj, M, F, csm, C, dcw);
    size_t nimg = (size_t)F;
    for (unsigned d = 0; d < D; d++) nimg *= (size_t)n[d];
    RecordingCg<complext<float>> cg(static_cast<char *>(iterates), nimg * sizeof(complext<float>));
    cg.set_encoding_operator(E);
    cg.set_max_iterations((unsigned)iterations);
    cg.set_tc_tolerance(tc_tolerance);
    auto d = upload<complext<float>>({(size_t)(M * F), (size_t)C}, data);
    auto x = cg.solve(&d);
    if (!x) throw std::runtime_error("cuCgSolver::solve returned no result");
    cuda_ok(cudaDeviceSynchronize(), "cg");
    download(*x, x_out);
    if (iterations_run) *iterations_run = cg.k_;
    return 0;
}

// Device time of fn() on the legacy default stream (the stream the
// reference runs on), averaged over reps after two warm-up calls.
template <class Fn> float time_ms(int reps, Fn &&fn) {
    for (int i = 0; i < 2; i++) fn();
    cudaEvent_t a, b;
    cuda_ok(cudaEventCreate(&a), "event");
    cuda_ok(cudaEventCreate(&b), "event");
    float total = 0.f;
    for (int i = 0; i < reps; i++) {
        cuda_ok(cudaEventRecord(a, 0), "record");
        fn();
        cuda_ok(cudaEventRecord(b, 0), "record");
        cuda_ok(cudaEventSynchronize(b), "sync");
        float ms = 0.f;
        cuda_ok(cudaEventElapsedTime(&ms, a, b), "elapsed");
        total += ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return total / (float)reps;
}

// Times one cuCgSolver::solve (E^H d and `iterations` iterations, everything
// the reference does per call) with the operator set up and preprocessed.
template <unsigned D>
int time_cg_sense(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
                  const void *csm, uint64_t C, const float *dcw, const void *data, int iterations, int reps,
                  float *ms) {
    auto E = make_sense<D>(n, mos, W, traj, M, F, csm, C, dcw);
    cuCgSolver<complext<float>> cg;
    cg.set_encoding_operator(E);
    cg.set_max_iterations((unsigned)iterations);
    cg.set_tc_tolerance(0.f);
    auto d = upload<complext<float>>({(size_t)(M * F), (size_t)C}, data);
    *ms = time_ms(reps, [&] { auto x = cg.solve(&d); (void)x; });
    return 0;
}

// Times compute(FORWARDS_C2NC) and compute(BACKWARDS_NC2C, dcw) on a
// preprocessed plan; also the preprocess itself.
template <unsigned D>
int time_nfft(const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M, uint64_t F,
              const void *img, const float *dcw, uint64_t B, int reps, float *ms_fwd, float *ms_adj,
              float *ms_prep) {
    auto plan = NFFT<cuNDArray, float, D>::make_plan(vec<D>(n), vec<D>(mos), W, ConvolutionType::STANDARD);
    auto t = upload_traj<D>(traj, M, F);
    *ms_prep = time_ms(reps, [&] { plan->preprocess(t, NFFT_prep_mode::ALL); });
    std::vector<size_t> im = dims_of<D>(n);
    im.push_back((size_t)F);
    im.push_back((size_t)B);
    auto x = upload<complext<float>>(im, img);
    cuNDArray<complext<float>> y(std::vector<size_t>{(size_t)M, (size_t)F, (size_t)B});
    cuNDArray<complext<float>> xb(im);
    cuNDArray<float> w;
    if (dcw) w = upload<float>({(size_t)M, (size_t)F}, dcw);
    *ms_fwd = time_ms(reps, [&] { plan->compute(x, y, nullptr, NFFT_comp_mode::FORWARDS_C2NC); });
    *ms_adj = time_ms(reps, [&] { plan->compute(y, xb, dcw ? &w : nullptr, NFFT_comp_mode::BACKWARDS_NC2C); });
    return 0;
}

template <class Fn> int guarded(Fn &&fn) {
    try {
        g_err.clear();
        return fn();
    } catch (const std::exception &e) {
        g_err = e.what();
    } catch (...) {
        g_err = "unknown exception";
    }
    cudaGetLastError();
    return 1;
}

#define GBREF_DISPATCH(D, CALL)                                                                  \
    switch (D) {                                                                                 \
    case 1: return CALL(1);                                                                      \
    case 2: return CALL(2);                                                                      \
    case 3: return CALL(3);                                                                      \
    default: throw std::runtime_error("D must be 1, 2 or 3");                                    \
    }

}  // namespace

extern "C" {

const char *gbref_last_error() { return g_err.c_str(); }

int gbref_nfft_compute(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                       uint64_t F, const void *in, void *out, const float *dcw, int mode, uint64_t B,
                       int oversampled_image, int conv_type) {
    return guarded([&]() -> int {
#define C_(d) nfft_compute<d>(n, mos, W, traj, M, F, in, out, dcw, mode, B, oversampled_image, conv_type)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_nfft_mult_MH_M(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                         uint64_t F, const void *in, void *out, const float *dcw, uint64_t B) {
    return guarded([&]() -> int {
#define C_(d) nfft_mult_MH_M<d>(n, mos, W, traj, M, F, in, out, dcw, B)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_nfft_convolve(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                        uint64_t F, const void *in, void *out, int conv, uint64_t B, int accumulate) {
    return guarded([&]() -> int {
#define C_(d) nfft_convolve<d>(n, mos, W, traj, M, F, in, out, conv, B, accumulate)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_nfft_fft_deapodize(int D, const uint64_t *n, const uint64_t *mos, float W, void *data, uint64_t FB,
                             int op, int do_scale) {
    return guarded([&]() -> int {
#define C_(d) nfft_fft_deapod<d>(n, mos, W, data, FB, op, do_scale)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_sense_mult(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                     uint64_t F, const void *csm, uint64_t C, const float *dcw, const void *in, void *out,
                     int adjoint) {
    return guarded([&]() -> int {
#define C_(d) sense_mult<d>(n, mos, W, traj, M, F, csm, C, dcw, in, out, adjoint)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_cg_sense(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                   uint64_t F, const void *csm, uint64_t C, const float *dcw, const void *data, void *x_out,
                   int iterations, float tc_tolerance, void *iterates, int *iterations_run) {
    return guarded([&]() -> int {
#define C_(d) cg_sense<d>(n, mos, W, traj, M, F, csm, C, dcw, data, x_out, iterations, tc_tolerance, \
                          iterates, iterations_run)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_time_cg_sense(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                        uint64_t F, const void *csm, uint64_t C, const float *dcw, const void *data, int iterations,
                        int reps, float *ms) {
    return guarded([&]() -> int {
#define C_(d) time_cg_sense<d>(n, mos, W, traj, M, F, csm, C, dcw, data, iterations, reps, ms)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

int gbref_time_nfft(int D, const uint64_t *n, const uint64_t *mos, float W, const float *traj, uint64_t M,
                    uint64_t F, const void *img, const float *dcw, uint64_t B, int reps, float *ms_fwd,
                    float *ms_adj, float *ms_prep) {
    return guarded([&]() -> int {
#define C_(d) time_nfft<d>(n, mos, W, traj, M, F, img, dcw, B, reps, ms_fwd, ms_adj, ms_prep)
        GBREF_DISPATCH(D, C_)
#undef C_
    });
}

}  // extern "C"
