// NUFFT plan operations (compute / mult_MH_M / convolve / fft / deapodize /
// trajectory gradient), the non-Cartesian SENSE operator and the CG solver.
//
// Reference call sequences restated (paths relative to the Gadgetron tree):
//   NFFT_plan::compute          toolboxes/nfft/NFFT.hpp:105-240
//   NFFT_plan::mult_MH_M        toolboxes/nfft/NFFT.hpp:90-102
//   cuNonCartesianSenseOperator toolboxes/mri/pmri/gpu/cuNonCartesianSenseOperator.cu:14-90
//   cgSolver                    toolboxes/solvers/cgSolver.h:105-390
//   relativeResidualTCB         toolboxes/solvers/cgCallback.h:56-104
//   cgPreconditioner            toolboxes/solvers/cgPreconditioner.h:24-39
//
// The CG solver keeps every scalar on the device: dot products and norms are
// accumulated in FP64 (per-block partials summed in a fixed order by the last
// block, so results are reproducible), alpha/beta are computed on the device,
// and no host synchronisation happens between iterations.  The whole solve
// can be captured into one CUDA graph and replayed.
#include <cmath>
#include <cstring>

#include "gb_dft.cuh"
#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

// ----------------------------------------------------------- workspaces ---

float2 *ensure_img_os(NufftPlan &p, int64_t nbf, cudaStream_t st) {
    const size_t need = (size_t)nbf * p.kp.G;
    const bool re = p.img_os.ensure(need);
    // The zeros outside the interior band must hold for this batch count's
    // outer-major layout (the band's address range depends on nbf).
    if (re || p.img_os_dirty || p.img_os_batches_zeroed < (size_t)nbf || (p.D >= 2 && p.img_os_nbf != nbf)) {
        GB_CUDA(cudaMemsetAsync(p.img_os.get(), 0, p.img_os.n * sizeof(float2), st));
        p.img_os_batches_zeroed = p.img_os.n / p.kp.G;
        p.img_os_dirty = false;
        p.img_os_nbf = nbf;
    }
    return p.img_os.get();
}

float2 *ensure_kgrid(NufftPlan &p, int64_t nbf) {
    p.kgrid.ensure((size_t)nbf * p.kp.G);
    return p.kgrid.get();
}

float2 *ensure_samp(NufftPlan &p, int nb) {
    // room for either sorted layout ([nb][M] or [M][il])
    p.samp_ws.ensure((size_t)il_stride_for(nb) * p.Mtot);
    return p.samp_ws.get();
}

static void exec_fft(NufftPlan &p, float2 *in, float2 *out, int nbf, int dir, cudaStream_t st) {
    cufftHandle h = plan_fft(p, nbf, st);
    GB_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(in), reinterpret_cast<cufftComplex *>(out), dir));
}

static void exec_pass(NufftPlan &p, FftPass pass, float2 *in, float2 *out, int nbf, int dir, cudaStream_t st) {
    cufftHandle h = plan_fft_om(p, nbf, pass, st);
    GB_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(in), reinterpret_cast<cufftComplex *>(out), dir));
}

// Layout of the plan's oversampled workspaces for nbf batches.  2D with the
// project-written passes: standard ([batch][y][x]) -- a column's points are
// one row apart, so the strided y pass stays inside each batch's plane (with
// the outer-major layout they are nbf rows apart: 2.4 MB for 64 frames x 12
// coils at 384^2, a span of 0.9 GB per column).  3D, and 2D under the cuFFT
// passes: outer-major (the interior band of the outer dimension is one
// contiguous run over all batches).
KLayout ws_layout(const NufftPlan &p, int64_t nbf) {
    if (p.D == 2 && fft_custom_ok(p)) return klayout_standard(p.kp);
    return p.D >= 2 ? klayout_outer(p.kp, nbf) : klayout_standard(p.kp);
}

// Project-written passes (fft_custom_ok).  Forward: the padded image is
// nonzero only inside the centred N box (band_only), so every pass reads only
// the box's extent along its axis; the outer pass writes `kg`.  2D: x pass
// over the band rows, y pass.  3D: x pass over the band rows of the band
// slices, y pass within the band slices, z pass.
static void fft_forward_custom(NufftPlan &p, float2 *pad, float2 *kg, int64_t nbf, bool inverse, bool band_only,
                               cudaStream_t st) {
    const KParams &k = p.kp;
    const int m0 = k.mos[0], m1 = k.mos[1];
    const int x0 = band_only ? (m0 - k.N[0]) / 2 : 0, nx = band_only ? k.N[0] : m0;
    const int y0 = band_only ? (m1 - k.N[1]) / 2 : 0, ny = band_only ? k.N[1] : m1;
    if (p.D == 2) {   // standard layout (ws_layout): plane b holds rows y of m0 points
        const int64_t G = k.G;
        fft_rows(p, m0, pad, pad, (int64_t)ny * nbf, ny, y0, G, x0, x0 + nx, 0, m0, inverse, st);
        fft_cols(p, m1, pad, kg, nbf * m0, m0, G, m0, y0, y0 + ny, 0, m1, inverse, st);
        return;
    }
    const int m2 = k.mos[2];
    const int z0 = band_only ? (m2 - k.N[2]) / 2 : 0, nz = band_only ? k.N[2] : m2;
    const int64_t plane = (int64_t)m1 * m0;
    const int64_t ncols = nbf * plane;
    float2 *band = pad + (int64_t)z0 * ncols;       // slices z0 .. z0+nz of every batch
    const int64_t nsl = (int64_t)nz * nbf;
    fft_rows(p, m0, band, band, nsl * ny, ny, y0, plane, x0, x0 + nx, 0, m0, inverse, st);
    fft_cols(p, m1, band, band, nsl * m0, m0, plane, m0, y0, y0 + ny, 0, m1, inverse, st);
    fft_cols(p, m2, pad, kg, ncols, ncols, 0, ncols, z0, z0 + nz, 0, m2, inverse, st);
}

// Adjoint direction in place on `kg`: the crop reads only the centred N box
// (band_only), so every pass writes only the box's extent along its axis.
// 2D: y pass, x pass over the band rows.  3D: z pass, y pass within the band
// slices, x pass over the band rows of the band slices.
static void fft_adjoint_custom(NufftPlan &p, float2 *kg, int64_t nbf, bool inverse, bool band_only,
                               cudaStream_t st) {
    const KParams &k = p.kp;
    const int m0 = k.mos[0], m1 = k.mos[1];
    const int x0 = band_only ? (m0 - k.N[0]) / 2 : 0, nx = band_only ? k.N[0] : m0;
    const int y0 = band_only ? (m1 - k.N[1]) / 2 : 0, ny = band_only ? k.N[1] : m1;
    if (p.D == 2) {   // standard layout (ws_layout)
        const int64_t G = k.G;
        fft_cols(p, m1, kg, kg, nbf * m0, m0, G, m0, 0, m1, y0, y0 + ny, inverse, st);
        fft_rows(p, m0, kg, kg, (int64_t)ny * nbf, ny, y0, G, 0, m0, x0, x0 + nx, inverse, st);
        return;
    }
    const int m2 = k.mos[2];
    const int z0 = band_only ? (m2 - k.N[2]) / 2 : 0, nz = band_only ? k.N[2] : m2;
    const int64_t plane = (int64_t)m1 * m0;
    const int64_t ncols = nbf * plane;
    fft_cols(p, m2, kg, kg, ncols, ncols, 0, ncols, 0, m2, z0, z0 + nz, inverse, st);
    float2 *band = kg + (int64_t)z0 * ncols;
    const int64_t nsl = (int64_t)nz * nbf;
    fft_cols(p, m1, band, band, nsl * m0, m0, plane, m0, 0, m1, y0, y0 + ny, inverse, st);
    fft_rows(p, m0, band, band, nsl * ny, ny, y0, plane, 0, m0, x0, x0 + nx, inverse, st);
}

// Forward FFT of the padded workspace `pad` into `kg`.  D >= 2: the inner
// pass runs in place over the interior band only (band_only; every other
// row/slice of `pad` is zero), then the outer pass writes `kg`.  D == 1: one
// out-of-place transform (pad's zero exterior is kept).
static void fft_forward_ws(NufftPlan &p, float2 *pad, float2 *kg, int nbf, int dir, bool band_only,
                           cudaStream_t st) {
    if (p.D < 2) {
        exec_fft(p, pad, kg, nbf, dir, st);
        return;
    }
    if (fft_custom_ok(p)) {
        fft_forward_custom(p, pad, kg, nbf, dir == CUFFT_INVERSE, band_only, st);
        return;
    }
    if (band_only) {
        float2 *band = pad + fft_band_offset(p, nbf);
        exec_pass(p, FFT_PASS_A_BAND, band, band, nbf, dir, st);
    } else {
        exec_pass(p, FFT_PASS_A_FULL, pad, pad, nbf, dir, st);
    }
    exec_pass(p, FFT_PASS_B, pad, kg, nbf, dir, st);
}

// In-place FFT of the gridded workspace `kg` for the crop: the outer pass over
// every column, then the inner pass over the interior band only (band_only)
// or everything.
static void fft_adjoint_ws(NufftPlan &p, float2 *kg, int nbf, int dir, bool band_only, cudaStream_t st) {
    if (p.D < 2) {
        exec_fft(p, kg, kg, nbf, dir, st);
        return;
    }
    if (fft_custom_ok(p)) {
        fft_adjoint_custom(p, kg, nbf, dir == CUFFT_INVERSE, band_only, st);
        return;
    }
    exec_pass(p, FFT_PASS_B, kg, kg, nbf, dir, st);
    if (band_only) {
        float2 *band = kg + fft_band_offset(p, nbf);
        exec_pass(p, FFT_PASS_A_BAND, band, band, nbf, dir, st);
    } else {
        exec_pass(p, FFT_PASS_A_FULL, kg, kg, nbf, dir, st);
    }
}

// Forward NUFFT into device sample buffer (layout chosen by caller).
// csm != null: image [F][NN] and nb = coils.
void nufft_forward(NufftPlan &p, const float2 *img, const float2 *csm, int nb, bool img_os,
                   float2 *samples, SampleLayout layout, const float *dcw, int dcw_pow,
                   bool accumulate, cudaStream_t st, const PUpdate *pu) {
    const int64_t nbf = (int64_t)nb * p.F;
    const KLayout kl = ws_layout(p, nbf);
    float2 *pad = ensure_img_os(p, nbf, st);
    float2 *kg = ensure_kgrid(p, nbf);
    launch_pad_forward(p, img, csm, pad, nb, img_os, st, &kl, pu);
    if (img_os) p.img_os_dirty = true;
    fft_forward_ws(p, pad, kg, (int)nbf, CUFFT_FORWARD, !img_os, st);
    launch_degrid(p, kg, samples, nb, layout, dcw, dcw_pow, true, accumulate, st, &kl);
}

// Adjoint NUFFT from samples.  csm != null: out image [F][NN], nb = coils.
void nufft_adjoint(NufftPlan &p, const float2 *samples, SampleLayout layout, const float *dcw,
                   const float2 *csm, int nb, float2 *img, bool img_os, bool accumulate, float weight,
                   int fft_dir, cudaStream_t st) {
    const int64_t nbf = (int64_t)nb * p.F;
    const KLayout kl = ws_layout(p, nbf);
    float2 *kg = ensure_kgrid(p, nbf);
    launch_grid(p, samples, kg, nb, layout, dcw, true, false, st, &kl);
    fft_adjoint_ws(p, kg, (int)nbf, fft_dir, !img_os, st);
    launch_crop_adjoint(p, kg, csm, img, nb, img_os, accumulate, weight, fft_dir == CUFFT_FORWARD, st, &kl);
}

// Normal operator A^H W^2 A on images (csm optional), samples stay in tile order.
void nufft_normal(NufftPlan &p, const float2 *img, const float2 *csm, int nb, const float *dcw,
                  float2 *out, bool accumulate, float weight, cudaStream_t st) {
    float2 *samp = ensure_samp(p, nb);
    const SampleLayout lay = normal_op_layout(p, nb);
    nufft_forward(p, img, csm, nb, false, samp, lay, dcw, 2, false, st);
    nufft_adjoint(p, samp, lay, nullptr, csm, nb, out, false, accumulate, weight, CUFFT_INVERSE, st);
}

// Device time of the two convolutions of E^H E (degridding with dcw^2 into
// the plan's sample workspace, gridding back into the k-space workspace),
// each launched `reps` times exactly as the normal operator launches them,
// on the plan's own workspaces.  Before every launch `flush_bytes` of
// `flush` are overwritten (cudaMemsetAsync) so that each one starts with a
// cold L2.  Averages in milliseconds.
void nufft_time_normal_convolutions(NufftPlan &p, int nb, const float *dcw, int reps, void *flush,
                                    size_t flush_bytes, float *ms_grid, float *ms_degrid, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    if (reps <= 0) fail(GB_ERR_INVALID_ARGUMENT, "reps must be positive");
    const int64_t nbf = (int64_t)nb * p.F;
    float2 *kg = ensure_kgrid(p, nbf);
    float2 *samp = ensure_samp(p, nb);
    launch_grid_prepare(p, nb, st);
    const KLayout kl = ws_layout(p, nbf);
    const SampleLayout lay = normal_op_layout(p, nb);
    GB_CUDA(cudaMemsetAsync(kg, 0, (size_t)nbf * p.kp.G * sizeof(float2), st));
    cudaEvent_t e0, e1;
    GB_CUDA(cudaEventCreate(&e0));
    GB_CUDA(cudaEventCreate(&e1));
    double tg = 0.0, td = 0.0;
    for (int r = 0; r < reps + 1; r++) {   // the first round warms up, untimed
        for (int which = 0; which < 2; which++) {
            if (flush && flush_bytes) GB_CUDA(cudaMemsetAsync(flush, r & 0xff, flush_bytes, st));
            GB_CUDA(cudaEventRecord(e0, st));
            if (which == 0)
                launch_degrid(p, kg, samp, nb, lay, dcw, 2, true, false, st, &kl);
            else
                launch_grid(p, samp, kg, nb, lay, nullptr, true, false, st, &kl);
            GB_CUDA(cudaEventRecord(e1, st));
            GB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            GB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r > 0) (which == 0 ? td : tg) += ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_grid = (float)(tg / reps);
    *ms_degrid = (float)(td / reps);
}

void nufft_compute(NufftPlan &p, const void *in, void *out, const float *dcw, gb_comp_mode mode,
                   int nb, bool image_os, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "NFFT_plan::compute: preprocess has not been called");
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "NULL input/output");
    if (nb <= 0) fail(GB_ERR_INVALID_ARGUMENT, "number of batches must be positive");
    const float2 *ci = static_cast<const float2 *>(in);
    float2 *co = static_cast<float2 *>(out);
    switch (mode) {
        case GB_FORWARDS_C2NC:
            nufft_forward(p, ci, nullptr, nb, image_os, co, LAYOUT_ORIGINAL, dcw, 1, false, st);
            break;
        case GB_BACKWARDS_NC2C:
            nufft_adjoint(p, ci, LAYOUT_ORIGINAL, dcw, nullptr, nb, co, image_os, false, 1.f, CUFFT_INVERSE, st);
            break;
        case GB_FORWARDS_NC2C:
            nufft_adjoint(p, ci, LAYOUT_ORIGINAL, dcw, nullptr, nb, co, image_os, false, 1.f, CUFFT_FORWARD, st);
            break;
        default:
            fail(GB_ERR_INVALID_ARGUMENT, "BACKWARDS_C2NC is not supported (the reference form passes swapped arguments)");
    }
}

void nufft_mult_MH_M(NufftPlan &p, const void *in, void *out, const float *dcw, int nb, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "NFFT_plan::mult_MH_M: preprocess has not been called");
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "NULL input/output");
    nufft_normal(p, static_cast<const float2 *>(in), nullptr, nb, dcw, static_cast<float2 *>(out), false, 1.f, st);
}

void nufft_convolve(NufftPlan &p, const void *in, void *out, gb_conv_mode mode, bool accumulate, int nb,
                    cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "NFFT_plan::convolve: preprocess has not been called");
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "NULL input/output");
    if (mode == GB_CONV_C2NC)
        launch_degrid(p, static_cast<const float2 *>(in), static_cast<float2 *>(out), nb, LAYOUT_ORIGINAL,
                      nullptr, 1, false, accumulate, st);
    else
        launch_grid(p, static_cast<const float2 *>(in), static_cast<float2 *>(out), nb, LAYOUT_ORIGINAL,
                    nullptr, false, accumulate, st);
}

void nufft_fft(NufftPlan &p, void *data, gb_fft_mode mode, bool do_scale, int nbf, cudaStream_t st) {
    if (!data || nbf <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid fft arguments");
    float2 *d = static_cast<float2 *>(data);
    launch_timeswitch_scale(p, d, nbf, 1.f, st);
    exec_fft(p, d, d, nbf, mode == GB_FFT_FORWARDS ? CUFFT_FORWARD : CUFFT_INVERSE, st);
    launch_timeswitch_scale(p, d, nbf, do_scale ? (float)(1.0 / std::sqrt((double)p.kp.G)) : 1.f, st);
}

void nufft_deapodize(NufftPlan &p, void *data, int nbf, cudaStream_t st) {
    if (!data || nbf <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid deapodize arguments");
    launch_deapodize_os(p, static_cast<float2 *>(data), nbf, st);
}

void nufft_traj_grad(NufftPlan &p, const float2 *img, const float2 *weights, const float *dcw, float *grad,
                     int nb, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const int64_t nbf = (int64_t)nb * p.F;
    const KLayout kl = ws_layout(p, nbf);
    float2 *pad = ensure_img_os(p, nbf, st);
    float2 *kg = ensure_kgrid(p, nbf);
    launch_pad_forward(p, img, nullptr, pad, nb, false, st, &kl);
    fft_forward_ws(p, pad, kg, (int)nbf, CUFFT_FORWARD, true, st);
    launch_traj_grad(p, kg, weights, nb, dcw, grad, true, st, &kl);
}

void nufft_traj_grad_from_grid(NufftPlan &p, const float2 *grid, const float2 *weights, float *grad, int nb,
                               cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    launch_traj_grad(p, grid, weights, nb, nullptr, grad, false, st);
}

// ---------------------------------------------------------------- SENSE ---

void sense_mult_M(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st) {
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "cuNonCartesianSenseOperator::mult_M : 0x0 input/output not accepted");
    if (!s.csm) fail(GB_ERR_INVALID_ARGUMENT, "csm not set");
    if (!s.plan.prepped) fail(GB_ERR_NOT_PREPROCESSED, "operator not preprocessed");
    nufft_forward(s.plan, static_cast<const float2 *>(in), s.csm, s.ncoils, false, static_cast<float2 *>(out),
                  LAYOUT_ORIGINAL, s.dcw, 1, accumulate, st);
}

void sense_mult_MH(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st) {
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "cuNonCartesianSenseOperator::mult_MH : 0x0 input/output not accepted");
    if (!s.csm) fail(GB_ERR_INVALID_ARGUMENT, "csm not set");
    if (!s.plan.prepped) fail(GB_ERR_NOT_PREPROCESSED, "operator not preprocessed");
    nufft_adjoint(s.plan, static_cast<const float2 *>(in), LAYOUT_ORIGINAL, s.dcw, s.csm, s.ncoils,
                  static_cast<float2 *>(out), false, accumulate, 1.f, CUFFT_INVERSE, st);
}

void sense_mult_MH_M(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st) {
    if (!in || !out) fail(GB_ERR_INVALID_ARGUMENT, "NULL input/output");
    if (!s.csm) fail(GB_ERR_INVALID_ARGUMENT, "csm not set");
    if (!s.plan.prepped) fail(GB_ERR_NOT_PREPROCESSED, "operator not preprocessed");
    nufft_normal(s.plan, static_cast<const float2 *>(in), s.csm, s.ncoils, s.dcw, static_cast<float2 *>(out),
                 accumulate, 1.f, st);
}

// ------------------------------------------------------------------- CG ---

// Device scalars.  The CG vector is cut into `nseg` segments that iterate
// independently (one per frame when frames are solved independently, a
// single segment for the reference's coupled solve): each segment has its own
// rq, rq0, alpha, beta and stop flag.
struct CgGlobal {
    double tol;
    int iters, hist_base, all_done, pad;
    unsigned int seg_ctr, pad2;
};

constexpr int kDotBlocks = 296;

__device__ __forceinline__ double2 block_reduce_d2(double2 v, double2 *sh) {
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : make_double2(0.0, 0.0);
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
    }
    return v;
}

// Per-segment reduction: blocks (blockIdx.x, seg) write their partial; the
// last block of the segment to arrive sums the segment's partials in a fixed
// order (bit-reproducible) and returns true in all its threads.  No block
// waits for another.
__device__ bool last_block_sum(double2 mine, double2 *partials, unsigned int *ctr, double2 *total) {
    __shared__ double2 sh[32];
    __shared__ int s_last;
    double2 *seg_part = partials + (size_t)blockIdx.y * gridDim.x;
    double2 v = block_reduce_d2(mine, sh);
    if (threadIdx.x == 0) {
        seg_part[blockIdx.x] = v;
        __threadfence();
        const unsigned int old = atomicAdd(ctr, 1u);
        s_last = (old == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double2 acc = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        const double2 q = __ldcg(&seg_part[b]);
        acc.x += q.x;
        acc.y += q.y;
    }
    __syncthreads();
    acc = block_reduce_d2(acc, sh);
    if (threadIdx.x == 0) *ctr = 0u;
    *total = acc;
    return true;
}

// last_block_sum for NV values per block (slots blockIdx * NV + v of the
// segment's partials), summed in the same fixed order.
template <int NV>
__device__ bool last_block_sum_v(const double2 (&mine)[NV], double2 *partials, unsigned int *ctr,
                                 double2 (&total)[NV]) {
    __shared__ double2 sh[32];
    __shared__ int s_last;
    double2 *seg_part = partials + (size_t)blockIdx.y * gridDim.x * NV;
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const double2 r = block_reduce_d2(mine[v], sh);
        __syncthreads();   // sh is reused by the next reduction
        if (threadIdx.x == 0) seg_part[(size_t)blockIdx.x * NV + v] = r;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int old = atomicAdd(ctr, 1u);
        s_last = (old == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int v = 0; v < NV; v++) {
        double2 acc = make_double2(0.0, 0.0);
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
            const double2 q = __ldcg(&seg_part[(size_t)b * NV + v]);
            acc.x += q.x;
            acc.y += q.y;
        }
        acc = block_reduce_d2(acc, sh);
        __syncthreads();
        total[v] = acc;   // meaningful in thread 0
    }
    if (threadIdx.x == 0) *ctr = 0u;
    return true;
}

// kappa R^H R p for the regulariser R = diag(reg) (reg null: R = I), as
// imageOperator::mult_MH_M forms it: (p * reg) * reg.
__device__ __forceinline__ float2 reg_term(float2 pv, const float *reg, int64_t e) {
    if (!reg) return pv;
    const float w = reg[e];
    return make_float2((pv.x * w) * w, (pv.y * w) * w);
}

// q = weight * crop(...) + kappa * R^H R p, then <p, q> per segment -> alpha = rq / <p, q>.
__global__ void k_cg_crop_dot(KParams k, KLayout kl, const float *deap, int deap_stride, float scale,
                              const float2 *__restrict__ grid, const float2 *__restrict__ csm, int nb, int F,
                              const float2 *__restrict__ p, float2 *__restrict__ q, float weight, float kappa,
                              const float *__restrict__ reg, CgSeg *segs, int64_t seg_len, double2 *partials) {
    CgSeg &S = segs[blockIdx.y];
    if (S.done) return;
    const int ox = (k.mos[0] - k.N[0]) >> 1, oy = (k.mos[1] - k.N[1]) >> 1, oz = (k.mos[2] - k.N[2]) >> 1;
    // Rows of N0 pixels: a block takes whole rows (index math once per row,
    // threads along x).
    const int rows_per_frame = k.N[1] * k.N[2];
    const int seg_rows = (int)(seg_len / k.N[0]);
    const int row0 = (int)blockIdx.y * seg_rows;
    double2 acc = make_double2(0.0, 0.0);
    for (int r = blockIdx.x; r < seg_rows; r += gridDim.x) {
        const int R = row0 + r;
        const int f = R / rows_per_frame;
        const int rem = R - f * rows_per_frame;
        const int z = rem / k.N[1], y = rem - (rem / k.N[1]) * k.N[1];
        const int gy = y + oy, gz = z + oz;
        float fyz = 1.f;
        if (k.D > 1) fyz = deap[deap_stride + y];
        if (k.D > 2) fyz *= deap[2 * deap_stride + z];
        const int64_t grow = (int64_t)gz * kl.s_z + (int64_t)gy * kl.s_y + ox;   // grid cell of x = 0
        const int64_t nrow = (int64_t)rem * k.N[0];                            // pixel of x = 0 in a frame
        const int64_t erow = (int64_t)R * k.N[0];
        for (int x = threadIdx.x; x < k.N[0]; x += blockDim.x) {
            const int gx = x + ox;
            float fac = deap[x] * fyz;
            if ((gx + gy + gz) & 1) fac = -fac;
            fac *= scale * weight;
            const int64_t g = grow + x, n = nrow + x, e = erow + x;
            float2 s = make_float2(0.f, 0.f);
#pragma unroll 8
            for (int b = 0; b < nb; b++) {
                const float2 v = grid[((int64_t)b * F + f) * kl.s_bf + g];
                const float2 c = csm[(int64_t)b * k.NN + n];
                const float vr = v.x * fac, vi = v.y * fac;
                s.x += vr * c.x + vi * c.y;
                s.y += vi * c.x - vr * c.y;
            }
            const float2 pv = p[e];
            const float2 rp = reg_term(pv, reg, e);
            s.x += kappa * rp.x;
            s.y += kappa * rp.y;
            q[e] = s;
            // conj(p) * q
            acc.x += (double)pv.x * s.x + (double)pv.y * s.y;
            acc.y += (double)pv.x * s.y - (double)pv.y * s.x;
        }
    }
    double2 tot;
    if (last_block_sum(acc, partials, &S.ctr_dot, &tot) && threadIdx.x == 0) {
        const double den = tot.x * tot.x + tot.y * tot.y;
        // alpha = rq / pq  (rq real), cgSolver.h:318
        S.alpha_re = S.rq * tot.x / den;
        S.alpha_im = -S.rq * tot.y / den;
    }
}

// x += alpha p ; r -= alpha q ; rq' = Re<r, P^2 r> ; beta = rq'/rq ; stop rule
// per segment; the last segment to finish records max(rq/rq0) in the history.
__global__ void k_cg_update(int64_t seg_len, float2 *__restrict__ x, float2 *__restrict__ r,
                            const float2 *__restrict__ p, const float2 *__restrict__ q,
                            const float *__restrict__ P, int64_t Pn, CgSeg *segs, CgGlobal *G,
                            double2 *partials, double *hist) {
    CgSeg &S = segs[blockIdx.y];
    const bool was_done = S.done != 0;
    double2 acc = make_double2(0.0, 0.0);
    if (!was_done) {
        const float ar = (float)S.alpha_re, ai = (float)S.alpha_im;
        const int64_t e0 = (int64_t)blockIdx.y * seg_len;
        for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < seg_len;
             l += (int64_t)gridDim.x * blockDim.x) {
            const int64_t e = e0 + l;
            const float2 pv = p[e], qv = q[e];
            float2 xv = x[e], rv = r[e];
            xv.x += ar * pv.x - ai * pv.y;
            xv.y += ar * pv.y + ai * pv.x;
            rv.x -= ar * qv.x - ai * qv.y;
            rv.y -= ar * qv.y + ai * qv.x;
            x[e] = xv;
            r[e] = rv;
            float w2 = 1.f;
            if (P) { const float w = P[e]; w2 = w * w; }
            acc.x += (double)rv.x * (double)(rv.x * w2) + (double)rv.y * (double)(rv.y * w2);
        }
    }
    double2 tot;
    if (last_block_sum(acc, partials, &S.ctr_upd, &tot) && threadIdx.x == 0) {
        if (!was_done) {
            const double rq_new = tot.x;
            S.beta = rq_new / S.rq;
            S.rq = rq_new;
            S.metric = rq_new / S.rq0;
            if (S.metric < G->tol) S.done = 1;
        }
        __threadfence();
        const unsigned int old = atomicAdd(&G->seg_ctr, 1u);
        if (old == gridDim.y - 1) {   // last segment of this iteration
            __threadfence();
            G->seg_ctr = 0u;
            if (!G->all_done) {
                double mx = 0.0;
                int all = 1;
                for (unsigned s = 0; s < gridDim.y; s++) {
                    const double m = *((volatile double *)&segs[s].metric);
                    mx = m > mx ? m : mx;
                    all &= (*((volatile int *)&segs[s].done) != 0);
                }
                if (hist) hist[G->hist_base + G->iters] = mx;
                G->iters += 1;
                if (all) G->all_done = 1;
            }
        }
    }
}

__device__ __forceinline__ float2 cmul2(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ------------------------------------------------ fused CG iteration tail ---
//
// One cooperative launch per iteration replaces crop/<p,q>, the x/r update +
// <r,P^2 r> and the next iteration's direction update + forward pad.  Blocks
// keep the same image rows through all phases, so the only exchange between
// blocks is the two segment sums, taken through a grid barrier; every block
// of a segment sums the segment's block partials in the same order, so all
// of them hold bit-identical scalars.  Arithmetic is that of k_cg_crop_dot,
// k_cg_update and the pad kernel with the direction update.

struct TailArgs {
    KParams k;
    KLayout kl;
    const float *deap;       // [D][deap_stride] image-domain deapodization
    int deap_stride;
    float scale;             // 1/sqrt(G)
    const float2 *kg;        // k-space workspace after the inverse FFT (band rows transformed)
    const float2 *csm;
    int nb, F;
    float2 *x, *r, *p, *q;
    const float *P;
    float weight, kappa;
    const float *reg;        // image regulariser diagonal (null: identity)
    CgSeg *segs;
    CgGlobal *G;
    double2 *part1, *part2;  // [nseg][gridDim.x]
    double *hist;
    unsigned int *bar;       // per segment: barrier arrival count, generation
    unsigned int *err;
    uint32_t spin_limit;     // polls of a barrier wait before giving up
    float2 *pad;             // next iteration's padded image (outer-major), or null after the last iteration
    int pad_full;            // 1: whole band lines with their zeros (a cuFFT pass follows); 0: interior only
    int seg_rows;            // image rows (of N0 pixels) per segment
};

// Barrier of the nblocks blocks of one segment (a cooperative launch: all
// blocks resident; segments share nothing, so each has its own counters).
// The wait is bounded: after spin_limit polls (2^26 by default, about 4 s) the
// block records the failure in bit 1 of *err and goes on.  Past such a
// timeout the barrier counters no longer match the launch's phases, so the
// host clears them before every solve, and the solve's values are void (the
// caller learns it from the error word).
__device__ void tail_grid_barrier(unsigned int *bar, unsigned int nblocks, unsigned int *err,
                                  uint32_t spin_limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vb = bar;
        const unsigned int gen = vb[1];
        __threadfence();
        const unsigned int arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == nblocks) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            for (uint32_t i = 0; vb[1] == gen; i++) {
                if (i >= spin_limit) {
                    atomicOr(err, 2u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// Sum of a segment's block partials in a fixed order (same result in every block).
__device__ double2 tail_segment_sum(const double2 *part, int nparts, double2 *sh) {
    double2 v = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
        const double2 t = __ldcg(&part[b]);
        v.x += t.x;
        v.y += t.y;
    }
    v = block_reduce_d2(v, sh);
    __shared__ double2 s_tot;
    if (threadIdx.x == 0) s_tot = v;
    __syncthreads();
    const double2 tot = s_tot;
    __syncthreads();
    return tot;
}

// TPP threads share a pixel in the coil sums of phases 1 and 3 (coils b = sub,
// sub + TPP, ...; the partial sums are combined by a shuffle): each thread's
// loads are then one round of TPP-times fewer coils, which halves the
// dependent-latency chain of a short tail (one image row per block).  Blocks
// are 256 * TPP threads.
template <int TPP>
__global__ void __launch_bounds__(256 * TPP, 4 / TPP) k_cg_tail(TailArgs t) {
    __shared__ double2 sh[32];
    const KParams &k = t.k;
    const int seg = blockIdx.y, nbx = gridDim.x;
    const unsigned int nblocks = gridDim.x;   // blocks of this segment
    unsigned int *bar = t.bar + 2 * seg;
    CgSeg &S = t.segs[seg];
    const bool was_done = S.done != 0;
    const double rq = S.rq, rq0 = S.rq0;
    const int ox = (k.mos[0] - k.N[0]) >> 1, oy = (k.mos[1] - k.N[1]) >> 1, oz = (k.mos[2] - k.N[2]) >> 1;
    const int rows_per_frame = k.N[1] * k.N[2];
    const int row0 = seg * t.seg_rows;
    auto row_coords = [&](int R, int &f, int &z, int &y, int &rem) {
        f = R / rows_per_frame;
        rem = R - f * rows_per_frame;
        z = rem / k.N[1];
        y = rem - z * k.N[1];
    };
    // The block's rows are blockIdx.x, blockIdx.x + nbx, ...; its threads run
    // over the (row, column) pairs of all of them, so that every thread has
    // work when a row is narrower than the block (the host keeps
    // seg_rows * mos[0] below 2^31).
    const int n0 = k.N[0];
    const int my_rows = (int)blockIdx.x < t.seg_rows ? (t.seg_rows - 1 - (int)blockIdx.x) / nbx + 1 : 0;
    const int my_elems = my_rows * n0;

    const int sub = (int)threadIdx.x % TPP;                           // coil phase of this thread
    const int px0 = (int)threadIdx.x / TPP, pxs = (int)blockDim.x / TPP;   // pixel lane, pixels per pass

    // Phase 1: q = weight * crop(kg) * conj(csm) summed + kappa p ; <p, q>.
    // (The pass loop is uniform across the block so that the TPP threads of a
    // pixel meet at the shuffle.)
    double2 acc = make_double2(0.0, 0.0);
    if (!was_done) {
        for (int l0 = 0; l0 < my_elems; l0 += pxs) {
            const int l = l0 + px0;
            const bool ok = l < my_elems;
            const int i = ok ? l / n0 : 0, x = ok ? l - i * n0 : 0;
            const int rr = (int)blockIdx.x + i * nbx;
            int f, z, y, rem;
            row_coords(row0 + rr, f, z, y, rem);
            const int gy = y + oy, gz = z + oz;
            float fyz = 1.f;
            if (k.D > 1) fyz = t.deap[t.deap_stride + y];
            if (k.D > 2) fyz *= t.deap[2 * t.deap_stride + z];
            const int64_t grow = (int64_t)gz * t.kl.s_z + (int64_t)gy * t.kl.s_y + ox;
            const int64_t nrow = (int64_t)rem * n0;
            const int64_t erow = (int64_t)(row0 + rr) * n0;
            const int gx = x + ox;
            float fac = t.deap[x] * fyz;
            if ((gx + gy + gz) & 1) fac = -fac;
            fac *= t.scale * t.weight;
            const int64_t g = grow + x, n = nrow + x, e = erow + x;
            float2 s = make_float2(0.f, 0.f);
            if (ok) {
#pragma unroll 8
                for (int b = sub; b < t.nb; b += TPP) {
                    const float2 v = t.kg[((int64_t)b * t.F + f) * t.kl.s_bf + g];
                    const float2 c = t.csm[(int64_t)b * k.NN + n];
                    const float vr = v.x * fac, vi = v.y * fac;
                    s.x += vr * c.x + vi * c.y;
                    s.y += vi * c.x - vr * c.y;
                }
            }
            if (TPP == 2) {
                s.x += __shfl_xor_sync(0xffffffffu, s.x, 1);
                s.y += __shfl_xor_sync(0xffffffffu, s.y, 1);
            }
            if (ok && sub == 0) {
                const float2 pv = t.p[e];
                const float2 rp = reg_term(pv, t.reg, e);
                s.x += t.kappa * rp.x;
                s.y += t.kappa * rp.y;
                t.q[e] = s;
                acc.x += (double)pv.x * s.x + (double)pv.y * s.y;
                acc.y += (double)pv.x * s.y - (double)pv.y * s.x;
            }
        }
    }
    acc = block_reduce_d2(acc, sh);
    if (threadIdx.x == 0) t.part1[(size_t)seg * nbx + blockIdx.x] = acc;
    tail_grid_barrier(bar, nblocks, t.err, t.spin_limit);

    // Phase 2: alpha = rq / <p,q> ; x += alpha p ; r -= alpha q ; <r, P^2 r>.
    const double2 pq = tail_segment_sum(t.part1 + (size_t)seg * nbx, nbx, sh);
    double alpha_re = 0.0, alpha_im = 0.0;
    acc = make_double2(0.0, 0.0);
    if (!was_done) {
        const double den = pq.x * pq.x + pq.y * pq.y;
        alpha_re = rq * pq.x / den;
        alpha_im = -rq * pq.y / den;
        const float ar = (float)alpha_re, ai = (float)alpha_im;
        for (int l = threadIdx.x; l < my_elems; l += blockDim.x) {
            const int i = l / n0, x = l - i * n0;
            const int rr = (int)blockIdx.x + i * nbx;
            {
                const int64_t e = (int64_t)(row0 + rr) * n0 + x;
                const float2 pv = t.p[e], qv = t.q[e];
                float2 xv = t.x[e], rv = t.r[e];
                xv.x += ar * pv.x - ai * pv.y;
                xv.y += ar * pv.y + ai * pv.x;
                rv.x -= ar * qv.x - ai * qv.y;
                rv.y -= ar * qv.y + ai * qv.x;
                t.x[e] = xv;
                t.r[e] = rv;
                float w2 = 1.f;
                if (t.P) { const float w = t.P[e]; w2 = w * w; }
                acc.x += (double)rv.x * (double)(rv.x * w2) + (double)rv.y * (double)(rv.y * w2);
            }
        }
    }
    acc = block_reduce_d2(acc, sh);
    if (threadIdx.x == 0) t.part2[(size_t)seg * nbx + blockIdx.x] = acc;
    tail_grid_barrier(bar, nblocks, t.err, t.spin_limit);

    // Phase 3: segment scalars, stop rule, history; then the direction update
    // p = beta p + P^2 r and the forward pad of p for the next iteration.
    const double2 rr2 = tail_segment_sum(t.part2 + (size_t)seg * nbx, nbx, sh);
    bool done_now = was_done;
    float beta = 0.f;
    if (!was_done) {
        const double rq_new = rr2.x;
        beta = (float)(rq_new / rq);
        done_now = (rq_new / rq0) < t.G->tol;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!was_done) {
            const double rq_new = rr2.x;
            S.alpha_re = alpha_re;
            S.alpha_im = alpha_im;
            S.beta = rq_new / rq;
            S.rq = rq_new;
            S.metric = rq_new / rq0;
            if (S.metric < t.G->tol) S.done = 1;
        }
        __threadfence();
        const unsigned int old = atomicAdd(&t.G->seg_ctr, 1u);
        if (old == gridDim.y - 1) {   // last segment of this iteration
            __threadfence();
            t.G->seg_ctr = 0u;
            if (!t.G->all_done) {
                double mx = 0.0;
                int all = 1;
                for (unsigned s = 0; s < gridDim.y; s++) {
                    const double m = *((volatile double *)&t.segs[s].metric);
                    mx = m > mx ? m : mx;
                    all &= (*((volatile int *)&t.segs[s].done) != 0);
                }
                if (t.hist) t.hist[t.G->hist_base + t.G->iters] = mx;
                t.G->iters += 1;
                if (all) t.G->all_done = 1;
            }
        }
    }
    if (!t.pad) return;
    // interior only when the FFT passes read nothing else
    const int gx0 = t.pad_full ? 0 : ox, gx1 = t.pad_full ? k.mos[0] : ox + n0;
    const int w3 = gx1 - gx0;
    const int my_pad = my_rows * w3;
    for (int l0 = 0; l0 < my_pad; l0 += pxs) {   // uniform across the block (the __syncwarp below)
        const bool ok = l0 + px0 < my_pad;
        const int l = ok ? l0 + px0 : 0;
        const int i = l / w3;
        const int rr = (int)blockIdx.x + i * nbx;
        int f, z, y, rem;
        row_coords(row0 + rr, f, z, y, rem);
        const int gy = y + oy, gz = z + oz;
        float fyz = t.scale;
        if (k.D > 1) fyz *= t.deap[t.deap_stride + y];
        if (k.D > 2) fyz *= t.deap[2 * t.deap_stride + z];
        const int64_t gline = (int64_t)gz * t.kl.s_z + (int64_t)gy * t.kl.s_y;
        const int64_t nrow = (int64_t)rem * n0;
        const int64_t erow = (int64_t)(row0 + rr) * n0;
        {
            const int gx = gx0 + (l - i * w3);
            const int x = gx - ox;
            const bool in = ok && x >= 0 && x < k.N[0];
            float fac = 0.f;
            float2 v = make_float2(0.f, 0.f);
            const int64_t e = erow + x;
            if (in) {
                v = t.p[e];
                if (!done_now) {
                    float2 rv = t.r[e];
                    if (t.P) { const float w = t.P[e]; const float w2 = w * w; rv.x *= w2; rv.y *= w2; }
                    v = make_float2(beta * v.x + rv.x, beta * v.y + rv.y);
                }
                fac = t.deap[x] * fyz;
                if ((gx + gy + gz) & 1) fac = -fac;
            }
            __syncwarp();   // the pixel's other threads have read p
            if (in && !done_now && sub == 0) t.p[e] = v;
            const int64_t g = gline + gx, n = nrow + x;
#pragma unroll 8
            for (int b = sub; b < t.nb && ok; b += TPP) {
                const float2 c = in ? cmul2(v, t.csm[(int64_t)b * k.NN + n]) : make_float2(0.f, 0.f);
                t.pad[((int64_t)b * t.F + f) * t.kl.s_bf + g] = make_float2(c.x * fac, c.y * fac);
            }
        }
    }
    if (k.D == 3 && t.pad_full) {
        // rows of the band slices outside the interior rows: zero (the band
        // FFT pass overwrote them)
        const int zrows = k.mos[1] - k.N[1];
        const int64_t lines = (int64_t)t.F * k.N[2] * zrows;
        const int64_t nblk = (int64_t)gridDim.x * gridDim.y, bid = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
        for (int64_t L = bid; L < lines; L += nblk) {
            const int j = (int)(L % zrows);
            const int64_t fz = L / zrows;
            const int z = (int)(fz % k.N[2]), f = (int)(fz / k.N[2]);
            const int gy = j < oy ? j : j + k.N[1], gz = z + oz;
            const int64_t gline = (int64_t)gz * t.kl.s_z + (int64_t)gy * t.kl.s_y;
            for (int b = 0; b < t.nb; b++)
                for (int gx = threadIdx.x; gx < k.mos[0]; gx += blockDim.x)
                    t.pad[((int64_t)b * t.F + f) * t.kl.s_bf + gline + gx] = make_float2(0.f, 0.f);
        }
    }
}

// ----------------------------------- CG with the row passes fused (2D) ---
//
// 2D plans under the project FFT passes run the CG iteration as plain
// launches with no grid barrier: the x (row) pass of each FFT direction is
// fused with what the iteration does next to it.  Short iterations (every row
// kernel one wave) fold the update into the next pad, as below: six launches.
// Long ones (many frames) keep k_cg_update after k_rows_crop_dot (x, r,
// <r, P^2 r>, beta, stop rule, history: its grid-stride loops move the CG
// vectors at full bandwidth) and k_rows_pad only updates p: seven launches.
//   k_rows_pad       the previous iteration's end -- x += alpha p, r -= alpha q,
//                    p = beta p + P^2 r for segments still running, the FP64
//                    partial of <r, P^2 r> and, in the segment's last block, the
//                    residual, stop rule and history (cgSolver.h:318-375) --
//                    then per coil the interior row p x csm x deapodization x
//                    checkerboard x 1/sqrt(G) transformed in place of the row
//                    pass's input: the padded image never goes through HBM;
//   (y pass, degridding, gridding, adjoint y pass: as in the other paths)
//   k_rows_crop_dot  per image row, every coil's band row transformed back,
//                    cropped in shared memory, deapodized and summed with
//                    conj(csm) into q (+ kappa R^2 p); the FP64 partials of
//                    <p, q>, <r, P^2 q> and <q, P^2 q>; the segment's last
//                    block sets alpha = rq / <p, q> and beta from
//                    rq' = rq - 2 Re(alpha <r, P^2 q>) + |alpha|^2 <q, P^2 q>,
//                    the norm of r - alpha q (float alpha, as the update uses
//                    it) expanded, so that k_rows_pad can update p in the same
//                    pass as r: the band rows of the adjoint never go through
//                    HBM and no separate update launch is needed.  rq itself
//                    is always the dot of the stored r (k_rows_pad, k_cg_init),
//                    so the expansion's rounding does not accumulate.
// After the last iteration k_cg_update applies the final x and r update.  A
// block is one image row of one frame (all coils: one half-warp per coil and
// round).  The arithmetic of every element is that of k_pad_forward /
// k_fft_rows / k_cg_crop_dot / k_cg_update (the same expressions and row
// transform); only beta's rounding differs (relative ~1e-7 of rq / rq').

struct RowsArgs {
    KParams k;
    const float *deap;   // [D][deap_stride] image-domain deapodization
    int deap_stride;
    float scale, weight, kappa;
    const float *reg;
    const float2 *csm;
    int nb, F;
    float2 *ws;          // k_rows_pad: the padded workspace (band rows written); k_rows_crop_dot: k-space (band rows read)
    const float2 *tw;    // W_N^e of the row length mos[0]
    float2 *x;
    float2 *p;
    float2 *r;
    float2 *q;
    const float *P;
    CgSeg *segs;
    CgGlobal *G;
    double *hist;
    double2 *partials;
    int update;          // k_rows_pad: 0 none, 1 p = beta p + P^2 r, 2 the previous iteration's whole end (x, r, p, residual)
    int expand;          // k_rows_crop_dot: also beta from the expanded |r - alpha q|^2 (with update 2)
    int crop_alias;      // k_rows_crop_dot: coil b's cropped row in half-warp b's exchange cells (one round)
};

template <int N2, int IN>
__global__ void __launch_bounds__(256) k_rows_pad(RowsArgs a) {
    extern __shared__ float2 rows_sm[];   // [half-warps][17 N2] exchange, then the row of p
    const KParams &k = a.k;
    const int N0 = k.N[0], N1 = k.N[1], m0 = k.mos[0];
    const int R = blockIdx.y * gridDim.x + blockIdx.x, f = R / N1, y = R - f * N1;
    const int ox = (m0 - N0) >> 1, oy = (k.mos[1] - N1) >> 1;
    const int gy = y + oy;
    const int hw = threadIdx.x >> 4, t = threadIdx.x & 15, nhw = blockDim.x >> 4;
    float2 *rs = rows_sm + hw * (17 * N2);
    float2 *prow = rows_sm + nhw * (17 * N2);
    CgSeg &S = a.segs[blockIdx.y];
    const bool was_done = S.done != 0;
    const int64_t erow = ((int64_t)f * N1 + y) * N0;
    double2 acc = make_double2(0.0, 0.0);
    const bool upd = a.update == 2 && !was_done;
    const bool upd_p = a.update == 1 && !was_done;
    const float ar = (float)S.alpha_re, ai = (float)S.alpha_im, beta = (float)S.beta;
    for (int x = threadIdx.x; x < N0; x += blockDim.x) {
        const int64_t e = erow + x;
        float2 v = a.p[e];
        if (upd_p) {   // p = beta p + P^2 r (beta from k_cg_update), in place
            float2 rv = a.r[e];
            if (a.P) { const float w = a.P[e]; const float w2 = w * w; rv.x *= w2; rv.y *= w2; }
            v = make_float2(beta * v.x + rv.x, beta * v.y + rv.y);
            a.p[e] = v;
        }
        if (upd) {
            // x += alpha p ; r -= alpha q  (as k_cg_update)
            const float2 qv = a.q[e];
            float2 xv = a.x[e], rv = a.r[e];
            xv.x += ar * v.x - ai * v.y;
            xv.y += ar * v.y + ai * v.x;
            rv.x -= ar * qv.x - ai * qv.y;
            rv.y -= ar * qv.y + ai * qv.x;
            a.x[e] = xv;
            a.r[e] = rv;
            float w2 = 1.f;
            if (a.P) { const float w = a.P[e]; w2 = w * w; }
            acc.x += (double)rv.x * (double)(rv.x * w2) + (double)rv.y * (double)(rv.y * w2);
            // p = beta p + P^2 r  (as the pad's direction update)
            if (a.P) { rv.x *= w2; rv.y *= w2; }
            v = make_float2(beta * v.x + rv.x, beta * v.y + rv.y);
            a.p[e] = v;
        }
        prow[x] = v;
    }
    // <r, P^2 r> of the updated r: the segment's last block records the
    // residual, stop rule and history (its reduction's barriers also make
    // the row of p visible to the transforms).
    if (a.update == 2) {
        double2 tot[1];
        const double2 mine[1] = {acc};
        if (last_block_sum_v<1>(mine, a.partials, &S.ctr_upd, tot) && threadIdx.x == 0) {
            if (!was_done) {   // residual, stop rule (cgSolver.h:336-352)
                const double rq_new = tot[0].x;
                S.rq = rq_new;
                S.metric = rq_new / S.rq0;
                if (S.metric < a.G->tol) S.done = 1;
            }
            __threadfence();
            const unsigned int old = atomicAdd(&a.G->seg_ctr, 1u);
            if (old == gridDim.y - 1) {   // last segment of this iteration: history
                __threadfence();
                a.G->seg_ctr = 0u;
                if (!a.G->all_done) {
                    double mx = 0.0;
                    int all = 1;
                    for (unsigned s = 0; s < gridDim.y; s++) {
                        const double m = *((volatile double *)&a.segs[s].metric);
                        mx = m > mx ? m : mx;
                        all &= (*((volatile int *)&a.segs[s].done) != 0);
                    }
                    if (a.hist) a.hist[a.G->hist_base + a.G->iters] = mx;
                    a.G->iters += 1;
                    if (all) a.G->all_done = 1;
                }
            }
        }
    }
    __syncthreads();
    float fyz = a.scale;
    fyz *= a.deap[a.deap_stride + y];
    for (int c0 = 0; c0 < a.nb; c0 += nhw) {   // uniform across the block
        const int b = c0 + hw;
        const bool ok = b < a.nb;
        const float2 *crow = a.csm + (int64_t)(ok ? b : 0) * k.NN + (int64_t)y * N0;
        float2 *orow = a.ws + ((int64_t)(ok ? b : 0) * a.F + f) * k.G + (int64_t)gy * m0;
        row_fft_halfwarp<N2, IN, kSpanAll>(
            t, 1.f, a.tw, rs, ox, ox + N0, 0, m0,
            [&](int o) {
                if (!ok) return make_float2(0.f, 0.f);
                const int x = o - ox;
                float fac = a.deap[x] * fyz;
                if ((o + gy) & 1) fac = -fac;
                const float2 c = cmul(prow[x], crow[x]);
                return make_float2(c.x * fac, c.y * fac);
            },
            [&](int kk, float2 v) {
                if (ok) orow[kk] = v;
            });
        __syncwarp();   // this half-warp's exchange is read before the next round writes it
    }
}

template <int N2, int OUT>
__global__ void __launch_bounds__(256, (N2 <= 24) ? 3 : 2) k_rows_crop_dot(RowsArgs a) {
    // [half-warps][17 N2] exchange, then [nb][N0] cropped rows; with
    // crop_alias (every coil in the first round, N0 <= 272) coil b's cropped
    // row takes the first N0 exchange cells of half-warp b, which the row
    // transform has read before it stores.
    extern __shared__ float2 rows_sm[];
    const KParams &k = a.k;
    const int N0 = k.N[0], N1 = k.N[1], m0 = k.mos[0];
    CgSeg &S = a.segs[blockIdx.y];
    if (S.done) return;   // the whole segment
    const int R = blockIdx.y * gridDim.x + blockIdx.x, f = R / N1, y = R - f * N1;
    const int ox = (m0 - N0) >> 1, oy = (k.mos[1] - N1) >> 1;
    const int gy = y + oy;
    const int hw = threadIdx.x >> 4, t = threadIdx.x & 15, nhw = blockDim.x >> 4;
    float2 *rs = rows_sm + hw * (17 * N2);
    float2 *crop = a.crop_alias ? rows_sm : rows_sm + nhw * (17 * N2);
    const int cst = a.crop_alias ? 17 * N2 : N0;   // crop row stride
    for (int c0 = 0; c0 < a.nb; c0 += nhw) {   // uniform across the block
        const int b = c0 + hw;
        const bool ok = b < a.nb;
        const float2 *irow = a.ws + ((int64_t)(ok ? b : 0) * a.F + f) * k.G + (int64_t)gy * m0;
        float2 *crow = crop + (int64_t)(ok ? b : 0) * cst - ox;
        row_fft_halfwarp<N2, kSpanAll, OUT>(
            t, -1.f, a.tw, rs, 0, m0, ox, ox + N0,
            [&](int o) { return ok ? irow[o] : make_float2(0.f, 0.f); },
            [&](int kk, float2 v) {
                if (ok) crow[kk] = v;
            });
        __syncwarp();
    }
    __syncthreads();
    // q = weight * crop * conj(csm) summed + kappa R^2 p ; <p, q>  (as k_cg_crop_dot)
    float fyz = 1.f;
    fyz = a.deap[a.deap_stride + y];
    const int64_t nrow = (int64_t)y * N0, erow = ((int64_t)f * N1 + y) * N0;
    double2 acc[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int x = threadIdx.x; x < N0; x += blockDim.x) {
        const int gx = x + ox;
        float fac = a.deap[x] * fyz;
        if ((gx + gy) & 1) fac = -fac;
        fac *= a.scale * a.weight;
        const int64_t n = nrow + x, e = erow + x;
        float2 s = make_float2(0.f, 0.f);
#pragma unroll 8
        for (int b = 0; b < a.nb; b++) {
            const float2 v = crop[(int64_t)b * cst + x];
            const float2 c = a.csm[(int64_t)b * k.NN + n];
            const float vr = v.x * fac, vi = v.y * fac;
            s.x += vr * c.x + vi * c.y;
            s.y += vi * c.x - vr * c.y;
        }
        const float2 pv = a.p[e];
        const float2 rp = reg_term(pv, a.reg, e);
        s.x += a.kappa * rp.x;
        s.y += a.kappa * rp.y;
        a.q[e] = s;
        // conj(p) q ; w conj(r) q ; w |q|^2   (w = P^2)
        acc[0].x += (double)pv.x * s.x + (double)pv.y * s.y;
        acc[0].y += (double)pv.x * s.y - (double)pv.y * s.x;
        if (a.expand) {
            const float2 rv = a.r[e];
            double w2 = 1.0;
            if (a.P) { const double w = a.P[e]; w2 = w * w; }
            acc[1].x += w2 * ((double)rv.x * s.x + (double)rv.y * s.y);
            acc[1].y += w2 * ((double)rv.x * s.y - (double)rv.y * s.x);
            acc[2].x += w2 * ((double)s.x * s.x + (double)s.y * s.y);
        }
    }
    if (!a.expand) {
        double2 tot;
        if (last_block_sum(acc[0], a.partials, &S.ctr_dot, &tot) && threadIdx.x == 0) {
            const double den = tot.x * tot.x + tot.y * tot.y;
            // alpha = rq / pq  (rq real), cgSolver.h:318
            S.alpha_re = S.rq * tot.x / den;
            S.alpha_im = -S.rq * tot.y / den;
        }
        return;
    }
    double2 tot[3];
    if (last_block_sum_v<3>(acc, a.partials, &S.ctr_dot, tot) && threadIdx.x == 0) {
        const double den = tot[0].x * tot[0].x + tot[0].y * tot[0].y;
        // alpha = rq / pq  (rq real), cgSolver.h:318
        const double rq = S.rq;
        S.alpha_re = rq * tot[0].x / den;
        S.alpha_im = -rq * tot[0].y / den;
        // |r - alpha q|^2_w with alpha as the update rounds it
        const double fr = (double)(float)S.alpha_re, fi = (double)(float)S.alpha_im;
        const double rq_new = rq - 2.0 * (fr * tot[1].x - fi * tot[1].y) + (fr * fr + fi * fi) * tot[2].x;
        S.beta = rq_new / rq;
    }
}

// Threads of the fused row kernels: one half-warp per coil and round, whole
// warps, at most 256 (coils beyond 16 take several rounds).
static int rows_threads(int nb) { return 32 * std::max(1, std::min(8, (nb + 1) / 2)); }

// Whether k_rows_crop_dot keeps coil b's cropped row in half-warp b's
// exchange cells: every coil in one round, and the row within the cells that
// the transform's first column group reads (272) when it has several groups.
static bool rows_crop_alias(const KParams &k, int nb, int threads) {
    return nb <= threads / 16 && (k.mos[0] / 16 <= 16 || k.N[0] <= 272);
}

static size_t rows_smem(const KParams &k, int nb, int threads, bool crop) {
    const size_t xch = (size_t)(threads / 16) * 17 * (k.mos[0] / 16);
    // crop: the cropped rows of every coil (unless they share the exchange
    // cells); pad: the row of p
    if (crop && rows_crop_alias(k, nb, threads)) return xch * sizeof(float2);
    return (xch + (crop ? (size_t)nb * k.N[0] : (size_t)k.N[0])) * sizeof(float2);
}

template <int N2, int SPAN>
static void launch_rows_pad_t(const RowsArgs &a, dim3 g, int threads, size_t smem, cudaStream_t st) {
    auto kern = k_rows_pad<N2, SPAN>;
    if (smem > 48 * 1024) GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, threads, smem, st>>>(a); ::gb::note_launch();
}

template <int N2, int SPAN>
static void launch_rows_crop_t(const RowsArgs &a, dim3 g, int threads, size_t smem, cudaStream_t st) {
    auto kern = k_rows_crop_dot<N2, SPAN>;
    if (smem > 48 * 1024) GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, threads, smem, st>>>(a); ::gb::note_launch();
}

#define GB_ROWS_N2_SWITCH(n2, CALL)                 \
    switch (n2) {                                   \
        case 2: CALL(2); break;                     \
        case 4: CALL(4); break;                     \
        case 6: CALL(6); break;                     \
        case 8: CALL(8); break;                     \
        case 10: CALL(10); break;                   \
        case 12: CALL(12); break;                   \
        case 16: CALL(16); break;                   \
        case 20: CALL(20); break;                   \
        case 24: CALL(24); break;                   \
        case 32: CALL(32); break;                   \
        case 40: CALL(40); break;                   \
        default: fail(GB_ERR_INTERNAL, "unsupported FFT length"); \
    }

// Whether the CG iteration runs with the fused row passes: 2D plans under the
// project FFT passes whose fused kernels fit in shared memory.
static bool rows_fused_ok(const NufftPlan &p, int nb) {
    if (p.D != 2 || !fft_custom_ok(p)) return false;
    const int th = rows_threads(nb);
    return rows_smem(p.kp, nb, th, true) <= 200 * 1024 && rows_smem(p.kp, nb, th, false) <= 200 * 1024;
}

static void launch_rows_pad(const RowsArgs &a, int nseg, cudaStream_t st) {
    const int threads = rows_threads(a.nb);
    const size_t smem = rows_smem(a.k, a.nb, threads, false);
    const int rows = a.F * a.k.N[1];
    const dim3 g((unsigned)(rows / nseg), (unsigned)nseg);
    const bool half = a.k.N[0] * 2 == a.k.mos[0];
#define GB_ROWS_PAD(K) \
    (half ? launch_rows_pad_t<K, kSpanHalf>(a, g, threads, smem, st) : launch_rows_pad_t<K, kSpanRange>(a, g, threads, smem, st))
    GB_ROWS_N2_SWITCH(a.k.mos[0] / 16, GB_ROWS_PAD)
#undef GB_ROWS_PAD
    GB_CUDA(cudaGetLastError());
}

static void launch_rows_crop_dot(const RowsArgs &args, int nseg, cudaStream_t st) {
    RowsArgs a = args;
    const int threads = rows_threads(a.nb);
    a.crop_alias = rows_crop_alias(a.k, a.nb, threads) ? 1 : 0;
    const size_t smem = rows_smem(a.k, a.nb, threads, true);
    const int rows = a.F * a.k.N[1];
    const dim3 g((unsigned)(rows / nseg), (unsigned)nseg);
    const bool half = a.k.N[0] * 2 == a.k.mos[0];
#define GB_ROWS_CROP(K) \
    (half ? launch_rows_crop_t<K, kSpanHalf>(a, g, threads, smem, st) : launch_rows_crop_t<K, kSpanRange>(a, g, threads, smem, st))
    GB_ROWS_N2_SWITCH(a.k.mos[0] / 16, GB_ROWS_CROP)
#undef GB_ROWS_CROP
    GB_CUDA(cudaGetLastError());
}

// Initialisation per segment: r = rhs - q (q optional), p = P^2 r,
// rq = Re<r, p>; set_rq0 also records rq0 and clears the iteration state
// (cgSolver.h:219-288).
__global__ void k_cg_init(int64_t seg_len, const float2 *__restrict__ rhs, const float2 *__restrict__ q,
                          float2 *__restrict__ x, const float2 *__restrict__ x0, float2 *__restrict__ r,
                          float2 *__restrict__ p, const float *__restrict__ P, int64_t Pn, CgSeg *segs,
                          CgGlobal *G, double2 *partials, int set_rq0, double tol, int hist_base) {
    CgSeg &S = segs[blockIdx.y];
    const int64_t e0 = (int64_t)blockIdx.y * seg_len;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < seg_len;
         l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = e0 + l;
        float2 rv = rhs[e];
        if (q) { const float2 qv = q[e]; rv.x -= qv.x; rv.y -= qv.y; }
        r[e] = rv;
        float w2 = 1.f;
        if (P) { const float w = P[e]; w2 = w * w; }
        const float2 pv = make_float2(rv.x * w2, rv.y * w2);
        p[e] = pv;
        if (set_rq0) x[e] = x0 ? x0[e] : make_float2(0.f, 0.f);
        acc.x += (double)rv.x * pv.x + (double)rv.y * pv.y;
    }
    double2 tot;
    if (last_block_sum(acc, partials, &S.ctr_init, &tot) && threadIdx.x == 0) {
        S.rq = tot.x;
        if (set_rq0) {
            S.rq0 = tot.x;
            S.done = 0;
            S.metric = 1.0;
            if (blockIdx.y == 0) {
                G->tol = tol;
                G->iters = 0;
                G->hist_base = hist_base;
                G->all_done = 0;
                G->seg_ctr = 0u;
            }
        }
    }
}

// Refinement bookkeeping in FP64: x64 += x (delta); rhs = rhs0 - q in double.
__global__ void k_refine_accumulate(int64_t n, double2 *__restrict__ x64, const float2 *__restrict__ dx,
                                    float2 *__restrict__ xf) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double2 v = x64[e];
        const float2 d = dx[e];
        v.x += d.x;
        v.y += d.y;
        x64[e] = v;
        xf[e] = make_float2((float)v.x, (float)v.y);
    }
}

__global__ void k_refine_residual(int64_t n, const float2 *__restrict__ rhs0, const float2 *__restrict__ q,
                                  float2 *__restrict__ rhs) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = rhs0[e], b = q[e];
        rhs[e] = make_float2((float)((double)a.x - (double)b.x), (float)((double)a.y - (double)b.y));
    }
}

__global__ void k_copy_f2(int64_t n, const float2 *__restrict__ a, float2 *__restrict__ b) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        b[e] = a[e];
}

static unsigned blocks_for(int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, kDotBlocks));
}

// Launch shape of the segmented CG kernels: (blocks per segment, segments).
static dim3 seg_grid(const CgSolver &cg) {
    const int64_t bx = std::max<int64_t>(1, std::min<int64_t>((cg.seg_len + 255) / 256,
                                                              std::max<int64_t>(1, kDotBlocks / cg.nseg)));
    return dim3((unsigned)bx, (unsigned)cg.nseg);
}

CgSolver::~CgSolver() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
}

// E^H E p -> q with the fused crop/dot kernel (used inside the iteration).
// update_p: first apply the previous iteration's direction update
// p = beta p + P^2 r (folded into the forward pad).
static void cg_normal_dot(CgSolver &cg, cudaStream_t st, bool update_p) {
    SenseOp &s = *cg.E;
    NufftPlan &p = s.plan;
    const int nb = s.ncoils;
    const int64_t nbf = (int64_t)nb * p.F;
    float2 *samp = ensure_samp(p, nb);
    PUpdate pu{cg.p.get(), cg.r.get(), cg.precond, cg.segs.get(), cg.nseg > 1 ? 1 : 0};
    const SampleLayout lay = normal_op_layout(p, nb);
    nufft_forward(p, cg.p.get(), s.csm, nb, false, samp, lay, s.dcw, 2, false, st,
                  update_p ? &pu : nullptr);
    float2 *kg = ensure_kgrid(p, nbf);
    const KLayout kl = ws_layout(p, nbf);
    launch_grid(p, samp, kg, nb, lay, nullptr, true, false, st, &kl);
    fft_adjoint_ws(p, kg, (int)nbf, CUFFT_INVERSE, true, st);
    k_cg_crop_dot<<<seg_grid(cg), 256, 0, st>>>(p.kp, kl, p.deap_img.get(), p.maxN,
                                                (float)(1.0 / std::sqrt((double)p.kp.G)), kg, s.csm, nb,
                                                (int)p.F, cg.p.get(), cg.q.get(), cg.weight, cg.kappa,
                                                cg.kappa != 0.f ? cg.reg : nullptr, cg.segs.get(),
                                                cg.seg_len, cg.partials.get()); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

// One iteration.  The direction update p = beta p + P^2 r of the previous
// iteration runs inside this iteration's forward pad (none after the last).
static void cg_iteration(CgSolver &cg, cudaStream_t st, double *hist, bool first) {
    NufftPlan &p = cg.E->plan;
    const int64_t n = (int64_t)p.F * p.kp.NN;
    cg_normal_dot(cg, st, !first);
    k_cg_update<<<seg_grid(cg), 256, 0, st>>>(cg.seg_len, cg.x.get(), cg.r.get(), cg.p.get(), cg.q.get(),
                                              cg.precond, n, cg.segs.get(), cg.G.get(), cg.partials.get(), hist); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

// Iteration with the fused tail: the padded p is already in the pad buffer
// (written by the previous iteration's tail, or by the solve's first pad).
static void cg_iteration_fused(CgSolver &cg, cudaStream_t st, double *hist, bool last) {
    SenseOp &s = *cg.E;
    NufftPlan &p = s.plan;
    const int nb = s.ncoils;
    const int64_t nbf = (int64_t)nb * p.F;
    const KLayout kl = ws_layout(p, nbf);
    float2 *pad = p.img_os.get();
    float2 *kg = ensure_kgrid(p, nbf);
    float2 *samp = ensure_samp(p, nb);
    fft_forward_ws(p, pad, kg, (int)nbf, CUFFT_FORWARD, true, st);
    const SampleLayout lay = normal_op_layout(p, nb);
    launch_degrid(p, kg, samp, nb, lay, s.dcw, 2, true, false, st, &kl);
    launch_grid(p, samp, kg, nb, lay, nullptr, true, false, st, &kl);
    fft_adjoint_ws(p, kg, (int)nbf, CUFFT_INVERSE, true, st);
    TailArgs ta{};
    ta.k = p.kp;
    ta.kl = kl;
    ta.deap = p.deap_img.get();
    ta.deap_stride = p.maxN;
    ta.scale = (float)(1.0 / std::sqrt((double)p.kp.G));
    ta.kg = kg;
    ta.csm = s.csm;
    ta.nb = nb;
    ta.F = (int)p.F;
    ta.x = cg.x.get();
    ta.r = cg.r.get();
    ta.p = cg.p.get();
    ta.q = cg.q.get();
    ta.P = cg.precond;
    ta.weight = cg.weight;
    ta.kappa = cg.kappa;
    ta.reg = cg.kappa != 0.f ? cg.reg : nullptr;
    ta.segs = cg.segs.get();
    ta.G = cg.G.get();
    ta.part1 = cg.partials.get();
    ta.part2 = cg.partials2.get();
    ta.hist = hist;
    ta.bar = cg.tail_bar.get();
    ta.err = p.err_flag.get();
    ta.spin_limit = cg.barrier_spin_limit ? cg.barrier_spin_limit : (1u << 26);
    ta.pad = last ? nullptr : pad;
    ta.pad_full = fft_custom_ok(p) ? 0 : 1;
    ta.seg_rows = (int)(cg.seg_len / p.kp.N[0]);
    void *args[] = {&ta};
    if (cg.tail_tpp == 2)
        GB_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg_tail<2>, cg.tail_grid, dim3(512), args, 0, st));
    else
        GB_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg_tail<1>, cg.tail_grid, dim3(256), args, 0, st));
    ::gb::note_launch();
}

// One iteration with the fused row passes (2D, project FFT passes): see the
// kernels k_rows_pad / k_rows_crop_dot.  `first`: p is already P^2 r (nothing
// of a previous iteration to finish before the pad).
static void cg_iteration_rows(CgSolver &cg, cudaStream_t st, double *hist, bool first) {
    SenseOp &s = *cg.E;
    NufftPlan &p = s.plan;
    const KParams &k = p.kp;
    const int nb = s.ncoils;
    const int64_t nbf = (int64_t)nb * p.F;
    const int64_t n = (int64_t)p.F * k.NN;
    const KLayout kl = ws_layout(p, nbf);
    float2 *pad = p.img_os.get();
    float2 *kg = ensure_kgrid(p, nbf);
    float2 *samp = ensure_samp(p, nb);
    const int m0 = k.mos[0], m1 = k.mos[1];
    const int y0 = (m1 - k.N[1]) / 2;
    RowsArgs ra{};
    ra.k = k;
    ra.deap = p.deap_img.get();
    ra.deap_stride = p.maxN;
    ra.scale = (float)(1.0 / std::sqrt((double)k.G));
    ra.weight = cg.weight;
    ra.kappa = cg.kappa;
    ra.reg = cg.kappa != 0.f ? cg.reg : nullptr;
    ra.csm = s.csm;
    ra.nb = nb;
    ra.F = (int)p.F;
    ra.tw = fft_twiddles(p, m0, st);
    ra.x = cg.x.get();
    ra.p = cg.p.get();
    ra.r = cg.r.get();
    ra.q = cg.q.get();
    ra.P = cg.precond;
    ra.segs = cg.segs.get();
    ra.G = cg.G.get();
    ra.hist = hist;
    ra.partials = cg.partials.get();
    // the previous iteration's updates + pad + x pass (forward) into the band rows of the pad buffer
    ra.ws = pad;
    ra.update = first ? 0 : (cg.rows_fold ? 2 : 1);
    ra.expand = cg.rows_fold ? 1 : 0;
    launch_rows_pad(ra, cg.nseg, st);
    fft_cols(p, m1, pad, kg, nbf * m0, m0, k.G, m0, y0, y0 + k.N[1], 0, m1, false, st);
    const SampleLayout lay = normal_op_layout(p, nb);
    launch_degrid(p, kg, samp, nb, lay, s.dcw, 2, true, false, st, &kl);
    launch_grid(p, samp, kg, nb, lay, nullptr, true, false, st, &kl);
    fft_cols(p, m1, kg, kg, nbf * m0, m0, k.G, m0, 0, m1, y0, y0 + k.N[1], true, st);
    // x pass (adjoint) + crop + conjugate coil sum + <p, q> -> alpha (and beta)
    ra.ws = kg;
    launch_rows_crop_dot(ra, cg.nseg, st);
    if (!cg.rows_fold) {
        k_cg_update<<<seg_grid(cg), 256, 0, st>>>(cg.seg_len, cg.x.get(), cg.r.get(), cg.p.get(), cg.q.get(),
                                                  cg.precond, n, cg.segs.get(), cg.G.get(), cg.partials.get(), hist); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
    }
}

// Applies E^H E (with weight and kappa) to `in` into `out` without the dot.
static void cg_apply_normal(CgSolver &cg, const float2 *in, float2 *out, cudaStream_t st) {
    SenseOp &s = *cg.E;
    nufft_normal(s.plan, in, s.csm, s.ncoils, s.dcw, out, false, cg.weight, st);
}

// One full solve of E^H E x = rhs (device rhs) from x0 (optional) into cg.x.
static void cg_solve_once(CgSolver &cg, const float2 *rhs, const float2 *x0, double *hist, int hist_base,
                          cudaStream_t st) {
    NufftPlan &p = cg.E->plan;
    const int64_t n = (int64_t)p.F * p.kp.NN;
    k_cg_init<<<seg_grid(cg), 256, 0, st>>>(cg.seg_len, rhs, nullptr, cg.x.get(), x0, cg.r.get(), cg.p.get(),
                                            cg.precond, n, cg.segs.get(), cg.G.get(), cg.partials.get(), 1,
                                            (double)cg.tol, hist_base); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
    if (x0) {
        cg_apply_normal(cg, x0, cg.q.get(), st);
        k_cg_init<<<seg_grid(cg), 256, 0, st>>>(cg.seg_len, cg.r.get(), cg.q.get(), cg.x.get(), x0, cg.r.get(),
                                                cg.p.get(), cg.precond, n, cg.segs.get(), cg.G.get(),
                                                cg.partials.get(), 0, (double)cg.tol, hist_base); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
    }
    if (cg.use_rows) {
        for (uint32_t it = 0; it < cg.iterations; it++) cg_iteration_rows(cg, st, hist, it == 0);
        if (cg.rows_fold) {   // the last iteration's x and r update, residual and history
            k_cg_update<<<seg_grid(cg), 256, 0, st>>>(cg.seg_len, cg.x.get(), cg.r.get(), cg.p.get(), cg.q.get(),
                                                      cg.precond, n, cg.segs.get(), cg.G.get(), cg.partials.get(), hist); ::gb::note_launch();
            GB_CUDA(cudaGetLastError());
        }
        return;
    }
    if (cg.use_tail && cg.iterations > 0) {
        SenseOp &s = *cg.E;
        const int64_t nbf = (int64_t)s.ncoils * p.F;
        const KLayout kl = ws_layout(p, nbf);
        float2 *pad = ensure_img_os(p, nbf, st);
        launch_pad_forward(p, cg.p.get(), s.csm, pad, s.ncoils, false, st, &kl);
        for (uint32_t it = 0; it < cg.iterations; it++) cg_iteration_fused(cg, st, hist, it + 1 == cg.iterations);
        return;
    }
    for (uint32_t it = 0; it < cg.iterations; it++) cg_iteration(cg, st, hist, it == 0);
}

static void cg_prepare(CgSolver &cg, cudaStream_t st) {
    SenseOp &s = *cg.E;
    NufftPlan &p = s.plan;
    const int64_t n = (int64_t)p.F * p.kp.NN;
    const int nb = s.ncoils;
    cg.x.ensure(n);
    cg.r.ensure(n);
    cg.p.ensure(n);
    cg.q.ensure(n);
    cg.rhs0.ensure(n);
    cg.rhs.ensure(n);
    cg.nseg = cg.independent_frames ? (int)p.F : 1;
    cg.seg_len = n / cg.nseg;
    const dim3 sg = seg_grid(cg);
    cg.partials.ensure((size_t)sg.x * sg.y);
    cg.partials2.ensure((size_t)sg.x * sg.y);
    if (cg.tail_bar.ensure(2 * (size_t)cg.nseg))
        GB_CUDA(cudaMemsetAsync(cg.tail_bar.get(), 0, cg.tail_bar.n * sizeof(unsigned int), st));
    // The fused iteration tail needs D >= 2 and all of its blocks resident at
    // once (cooperative launch).
    cg.use_tail = false;
    cg.use_rows = cg.row_fusion && rows_fused_ok(p, nb) && cg.seg_len % p.kp.N[0] == 0;
    if (cg.use_rows) {
        // one block per image row in the row kernels: three partial slots each
        cg.partials.ensure(std::max<size_t>((size_t)sg.x * sg.y, 3 * (size_t)p.F * p.kp.N[1]));
        // A short iteration (every row kernel one wave: at most two rows per
        // SM) is bound by its chain of launches: the update then rides in the
        // next pad (six launches).  Long ones keep the separate update kernel,
        // whose grid-stride loops move x, r, p at full bandwidth.
        int dev = 0, nsm = 0;
        GB_CUDA(cudaGetDevice(&dev));
        GB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        cg.rows_fold = (int64_t)p.F * p.kp.N[1] <= 2 * (int64_t)nsm;
    }
    if (!cg.use_rows && p.D >= 2 && cg.seg_len % p.kp.N[0] == 0) {
        int dev = 0, coop = 0, nsm = 0, per_sm = 0;
        GB_CUDA(cudaGetDevice(&dev));
        GB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        GB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        // Two threads per pixel when every block holds at most one image row
        // (a short tail whose time is its latency chain); one otherwise (long
        // tails keep the larger number of resident blocks per segment).
        int per2 = 0;
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_cg_tail<2>, 512, 0));
        const int64_t rows = (cg.seg_len / p.kp.N[0]) * cg.nseg;
        cg.tail_tpp = (nb >= 8 && rows <= (int64_t)per2 * nsm) ? 2 : 1;
        if (cg.tail_tpp == 2)
            per_sm = per2;
        else
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_tail<1>, 256, 0));
        // blocks per segment: up to the resident capacity, at most one per image row
        const int64_t cap = (int64_t)per_sm * nsm;
        const int64_t seg_rows = cg.seg_len / p.kp.N[0];
        const int64_t bx = std::min<int64_t>(seg_rows, cap / cg.nseg);
        cg.use_tail = coop != 0 && bx >= 1 && seg_rows * (int64_t)p.kp.mos[0] < (int64_t)INT32_MAX;
        if (cg.use_tail) {
            cg.tail_grid = dim3((unsigned)bx, (unsigned)cg.nseg);
            cg.partials.ensure((size_t)bx * cg.nseg);
            cg.partials2.ensure((size_t)bx * cg.nseg);
        }
    }
    if (cg.segs.ensure(cg.nseg)) GB_CUDA(cudaMemsetAsync(cg.segs.get(), 0, cg.segs.n * sizeof(CgSeg), st));
    if (cg.G.ensure(1)) GB_CUDA(cudaMemsetAsync(cg.G.get(), 0, sizeof(CgGlobal), st));
    if (cg.refinements > 1) cg.x64.ensure(n);
    // Workspaces and FFT plans must exist before any graph capture.
    ensure_img_os(p, (int64_t)nb * p.F, st);
    ensure_kgrid(p, (int64_t)nb * p.F);
    ensure_samp(p, nb);
    plan_fft(p, nb * (int)p.F, st);
    if (p.D >= 2 && fft_custom_ok(p))   // twiddle tables are made outside stream capture
        fft_custom_prepare(p, st);
    else if (p.D >= 2)                  // and so are cuFFT plans
        for (FftPass pass : {FFT_PASS_A_BAND, FFT_PASS_A_FULL, FFT_PASS_B}) plan_fft_om(p, nb * (int)p.F, pass, st);
    // Split-tile counters/partials for the gridding kernel.
    launch_grid_prepare(p, nb, st);
}

static void cg_record(CgSolver &cg, const float2 *d, float2 *x_out, double *hist, cudaStream_t st) {
    SenseOp &s = *cg.E;
    NufftPlan &p = s.plan;
    const int64_t n = (int64_t)p.F * p.kp.NN;
    // A grid barrier that timed out in an earlier solve leaves its counters
    // out of step: start every solve from cleared ones.
    if (cg.use_tail) GB_CUDA(cudaMemsetAsync(cg.tail_bar.get(), 0, 2 * (size_t)cg.nseg * sizeof(unsigned int), st));
    // rhs0 = weight * E^H d
    nufft_adjoint(p, d, LAYOUT_ORIGINAL, s.dcw, s.csm, s.ncoils, cg.rhs0.get(), false, false, cg.weight,
                  CUFFT_INVERSE, st);
    if (cg.refinements <= 1) {
        cg_solve_once(cg, cg.rhs0.get(), cg.x0, hist, 0, st);
        k_copy_f2<<<blocks_for(n), 256, 0, st>>>(n, cg.x.get(), x_out); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        return;
    }
    GB_CUDA(cudaMemsetAsync(cg.x64.get(), 0, n * sizeof(double2), st));
    for (uint32_t k = 0; k < cg.refinements; k++) {
        const float2 *rhs = cg.rhs0.get();
        if (k > 0) {
            cg_apply_normal(cg, x_out, cg.q.get(), st);
            k_refine_residual<<<blocks_for(n), 256, 0, st>>>(n, cg.rhs0.get(), cg.q.get(), cg.rhs.get()); ::gb::note_launch();
            GB_CUDA(cudaGetLastError());
            rhs = cg.rhs.get();
        }
        cg_solve_once(cg, rhs, (k == 0) ? cg.x0 : nullptr, hist, (int)(k * cg.iterations), st);
        k_refine_accumulate<<<blocks_for(n), 256, 0, st>>>(n, cg.x64.get(), cg.x.get(), x_out); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
    }
}

void cg_solve(CgSolver &cg, const void *d, void *x_out, double *hist, uint32_t *iters_run, cudaStream_t st) {
    if (!cg.E) fail(GB_ERR_INVALID_ARGUMENT, "Error: cgSolver::compute_rhs : no encoding operator is set");
    if (!d || !x_out) fail(GB_ERR_INVALID_ARGUMENT, "NULL data or result");
    SenseOp &s = *cg.E;
    if (!s.csm) fail(GB_ERR_INVALID_ARGUMENT, "csm not set");
    if (!s.plan.prepped) fail(GB_ERR_NOT_PREPROCESSED, "operator not preprocessed");
    if (cg.kappa != 0.f && (cg.refinements > 1 || cg.x0))
        fail(GB_ERR_INVALID_ARGUMENT, "regularisation cannot be combined with x0 or refinement");
    NufftPlan &p = s.plan;
    const int64_t n = (int64_t)p.F * p.kp.NN;
    const float2 *dd = static_cast<const float2 *>(d);
    float2 *xo = static_cast<float2 *>(x_out);
    if (cg.iterations == 0) {
        nufft_adjoint(p, dd, LAYOUT_ORIGINAL, s.dcw, s.csm, s.ncoils, xo, false, false, cg.weight, CUFFT_INVERSE, st);
        if (iters_run) *iters_run = 0;
        return;
    }
    cg_prepare(cg, st);
    if (cg.use_graph) {
        GraphKey key{d, x_out, hist, cg.iterations, cg.refinements, cg.x0, cg.precond, cg.reg, cg.kappa, cg.weight,
                     cg.tol, s.csm, s.dcw, s.ncoils, plan_layout_signature(s.plan, s.ncoils * (int)s.plan.F),
                     cg.independent_frames, cg.barrier_spin_limit, cg.row_fusion};
        if (!cg.graph_exec || !(key == cg.graph_key)) {
            cudaStream_t cs;
            GB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            GB_CUDA(cudaStreamSynchronize(st));
            cudaGraph_t g;
            const uint64_t before = launch_count();
            GB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            try {
                cg_record(cg, dd, xo, hist, cs);
                cg.graph_kernels = launch_count() - before;
                note_launch(0 - cg.graph_kernels);   // captured, not launched
            } catch (...) {
                cudaGraph_t tmp;
                cudaStreamEndCapture(cs, &tmp);
                if (tmp) cudaGraphDestroy(tmp);
                cudaStreamDestroy(cs);
                throw;
            }
            GB_CUDA(cudaStreamEndCapture(cs, &g));
            if (cg.graph_exec) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(cg.graph_exec, g, &info) != cudaSuccess) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(cg.graph_exec);
                    cg.graph_exec = nullptr;
                }
            }
            if (!cg.graph_exec) GB_CUDA(cudaGraphInstantiate(&cg.graph_exec, g, 0));
            cudaGraphDestroy(g);
            GB_CUDA(cudaStreamDestroy(cs));
            // cuFFT plans were bound to the capture stream; rebind lazily.
            cg.graph_key = key;
        }
        GB_CUDA(cudaGraphLaunch(cg.graph_exec, st));
        note_launch(cg.graph_kernels);
    } else {
        cg_record(cg, dd, xo, hist, st);
    }
    CgGlobal hs;
    GB_CUDA(cudaMemcpyAsync(&hs, cg.G.get(), sizeof(CgGlobal), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    if (iters_run) *iters_run = (uint32_t)(hs.hist_base + hs.iters);
    (void)n;
}

}  // namespace gb
