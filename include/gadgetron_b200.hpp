// C++ host interface over the gadgetron_b200 C ABI, mirroring the reference
// classes the path sits behind:
//   NFFT<cuNDArray,float,D>::make_plan / NFFT_plan   (toolboxes/nfft/NFFT.h:54-175,
//                                                    toolboxes/nfft/gpu/cuNFFT.h:113-121)
//   cuNonCartesianSenseOperator<float,D>              (toolboxes/mri/pmri/gpu/cuNonCartesianSenseOperator.h:12-41)
//   cuCgSolver<float_complext>                        (toolboxes/solvers/gpu/cuCgSolver.h:24-29)
// Same method names and argument meaning; errors throw std::runtime_error as
// the reference does.  Arrays are raw device pointers (complex data as
// interleaved float pairs) with the reference's x-fastest layouts; a
// Gadgetron-side adapter wraps cuNDArray::get_data_ptr() around these calls.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "gadgetron_b200.h"

namespace gadgetron_b200 {

enum class NFFT_comp_mode { FORWARDS_C2NC = 0, FORWARDS_NC2C = 1, BACKWARDS_C2NC = 2, BACKWARDS_NC2C = 3 };
enum class NFFT_prep_mode { C2NC = 0, NC2C = 1, ALL = 2 };
enum class NFFT_conv_mode { C2NC = 0, NC2C = 1 };
enum class NFFT_fft_mode { FORWARDS = 0, BACKWARDS = 1 };

inline void check(gb_status s) {
    if (s != GB_OK) throw std::runtime_error(std::string("gadgetron_b200: ") + gb_last_error_message());
}

template <unsigned D>
class cuNFFT_plan {
public:
    cuNFFT_plan(const uint64_t (&matrix_size)[D], const uint64_t (&matrix_size_os)[D], float W,
                uint32_t flags = 0) {
        check(gb_nufft_plan_create((int)D, matrix_size, matrix_size_os, W, flags, &h_));
        for (unsigned d = 0; d < D; d++) {
            n_[d] = matrix_size[d];
            mos_[d] = matrix_size_os[d];
        }
        W_ = W;
    }
    ~cuNFFT_plan() { gb_nufft_plan_destroy(h_); }
    cuNFFT_plan(const cuNFFT_plan &) = delete;
    cuNFFT_plan &operator=(const cuNFFT_plan &) = delete;

    // preprocess(trajectory, mode): trajectory = num_samples D-vectors on the device.
    void preprocess(const float *trajectory, uint64_t num_samples, uint32_t num_frames = 1,
                    NFFT_prep_mode mode = NFFT_prep_mode::ALL, const uint64_t *frame_offsets = nullptr,
                    void *stream = nullptr) {
        check(gb_nufft_preprocess(h_, trajectory, num_samples, num_frames, frame_offsets, (gb_prep_mode)mode,
                                  stream));
    }
    void compute(const void *in, void *out, const float *dcw, NFFT_comp_mode mode, uint32_t num_batches = 1,
                 bool image_oversampled = false, void *stream = nullptr) {
        check(gb_nufft_compute(h_, in, out, dcw, (gb_comp_mode)mode, num_batches, image_oversampled ? 1 : 0,
                               stream));
    }
    void mult_MH_M(const void *in, void *out, const float *dcw, uint32_t num_batches = 1, void *stream = nullptr) {
        check(gb_nufft_mult_MH_M(h_, in, out, dcw, num_batches, stream));
    }
    void convolve(const void *in, void *out, NFFT_conv_mode mode, bool accumulate = false,
                  uint32_t num_batches = 1, void *stream = nullptr) {
        check(gb_nufft_convolve(h_, in, out, (gb_conv_mode)mode, accumulate ? 1 : 0, num_batches, stream));
    }
    void fft(void *data, NFFT_fft_mode mode, bool do_scale = true, uint32_t num_arrays = 1, void *stream = nullptr) {
        check(gb_nufft_fft(h_, data, (gb_fft_mode)mode, do_scale ? 1 : 0, num_arrays, stream));
    }
    void deapodize(void *image, bool fourier_domain = false, uint32_t num_arrays = 1, void *stream = nullptr) {
        check(gb_nufft_deapodize(h_, image, fourier_domain ? 1 : 0, num_arrays, stream));
    }
    const uint64_t *get_matrix_size() const { return n_; }
    const uint64_t *get_matrix_size_os() const { return mos_; }
    float get_W() const { return W_; }
    gb_nufft_plan handle() const { return h_; }

private:
    gb_nufft_plan h_ = nullptr;
    uint64_t n_[D]{}, mos_[D]{};
    float W_ = 0.f;
};

template <unsigned D>
class cuNonCartesianSenseOperator {
public:
    cuNonCartesianSenseOperator() = default;
    ~cuNonCartesianSenseOperator() { gb_sense_destroy(h_); }
    cuNonCartesianSenseOperator(const cuNonCartesianSenseOperator &) = delete;
    cuNonCartesianSenseOperator &operator=(const cuNonCartesianSenseOperator &) = delete;

    void setup(const uint64_t (&matrix_size)[D], const uint64_t (&matrix_size_os)[D], float W, uint32_t flags = 0) {
        if (h_) gb_sense_destroy(h_);
        h_ = nullptr;
        check(gb_sense_create((int)D, matrix_size, matrix_size_os, W, flags, &h_));
    }
    void preprocess(const float *trajectory, uint64_t num_samples, uint32_t num_frames = 1,
                    const uint64_t *frame_offsets = nullptr, void *stream = nullptr) {
        check(gb_sense_preprocess(h_, trajectory, num_samples, num_frames, frame_offsets, stream));
    }
    void set_csm(const void *csm, uint32_t num_coils) { check(gb_sense_set_csm(h_, csm, num_coils)); }
    void set_dcw(const float *dcw) { check(gb_sense_set_dcw(h_, dcw)); }
    void mult_M(const void *in, void *out, bool accumulate = false, void *stream = nullptr) {
        check(gb_sense_mult_M(h_, in, out, accumulate ? 1 : 0, stream));
    }
    void mult_MH(const void *in, void *out, bool accumulate = false, void *stream = nullptr) {
        check(gb_sense_mult_MH(h_, in, out, accumulate ? 1 : 0, stream));
    }
    void mult_MH_M(const void *in, void *out, bool accumulate = false, void *stream = nullptr) {
        check(gb_sense_mult_MH_M(h_, in, out, accumulate ? 1 : 0, stream));
    }
    void set_weight(float w) { weight_ = w; }
    float get_weight() const { return weight_; }
    gb_sense_op handle() const { return h_; }

private:
    gb_sense_op h_ = nullptr;
    float weight_ = 1.f;
};

class cuCgSolver {
public:
    cuCgSolver() { check(gb_cg_create(&h_)); }
    ~cuCgSolver() { gb_cg_destroy(h_); }
    cuCgSolver(const cuCgSolver &) = delete;
    cuCgSolver &operator=(const cuCgSolver &) = delete;

    template <unsigned D>
    void set_encoding_operator(cuNonCartesianSenseOperator<D> &E) {
        check(gb_cg_set_encoding_operator(h_, E.handle(), E.get_weight()));
    }
    void set_max_iterations(uint32_t n) { check(gb_cg_set_max_iterations(h_, n)); iterations_ = n; }
    void set_tc_tolerance(float t) { check(gb_cg_set_tc_tolerance(h_, t)); }
    void set_x0(const void *x0) { check(gb_cg_set_x0(h_, x0)); }
    void set_preconditioner(const float *weights) { check(gb_cg_set_preconditioner(h_, weights)); }
    void set_use_graph(bool on) { check(gb_cg_set_use_graph(h_, on ? 1 : 0)); }
    void set_frame_independent(bool on) { check(gb_cg_set_frame_independent(h_, on ? 1 : 0)); }
    void set_refinements(uint32_t n) { check(gb_cg_set_refinements(h_, n)); }

    // solve(d) -> x (written to x_out); returns the number of iterations run.
    uint32_t solve(const void *d, void *x_out, double *residual_history = nullptr, void *stream = nullptr) {
        uint32_t its = 0;
        check(gb_cg_solve(h_, d, x_out, residual_history, &its, stream));
        return its;
    }

private:
    gb_cg_solver h_ = nullptr;
    uint32_t iterations_ = 10;
};

}  // namespace gadgetron_b200
