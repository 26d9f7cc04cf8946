// Iterative density compensation estimate with a Jinc-shaped kernel
// (estimate_dcw, toolboxes/mri/sdc/SDC.hpp:19-80 and gpu/cuSDC.cu): starting
// from w = 1 (or the caller's weights), `iterations` times
//     grid = NC2C(w)            (gridding of the real weights),
//     t    = C2NC(grid)         (degridding back to the samples),
//     w    = t == 0 ? 0 : w / t
// on an oversampled grid of size round_up_32(N * os_factor) per dimension.
//
// The kernel is JincKernel (toolboxes/nfft/ConvolutionKernel.{h,hpp}):
// radius R = 0.96960938 * kernel_width, width 2R; the weight of a cell at
// offset u from the sample is 0 if any |u_d| > R, else with
// r = sqrt(sum u_d^2) / R: 0 if r >= 0.96960938, else the reference's
// degree-5 polynomial fit sum c_k r^k clipped at 0.  Cells and coordinates
// follow the gridding convention of the KB path: s = k mos + mos / 2 (float,
// as fma(k, mos, (mos + pad) / 2) - pad / 2 with pad = 2 ceil(R)), taps
// [ceil(s - R), floor(s + R)] per dimension, periodic wrap.
//
// It is a setup computation (once per trajectory), so the gridding here is a
// per-sample scatter with float atomics (the sum order per cell is not fixed,
// unlike the CG-loop gridding) and the degridding a per-sample gather.  A warp
// serves one sample, its lanes spread over the footprint's taps (up to 11^D
// at width 5.5, each with a square root, a division and a degree-5 polynomial), so
// that the tap arithmetic fills the SMs; the degridding sums the lanes'
// partial sums in a fixed butterfly order.  The grid and the trajectory-range
// flag are kept per device between calls.
#include <cmath>

#include "gb_internal.cuh"

namespace gb {

namespace {

// JincKernel constants (the reference's polynomial fit and normalised radius;
// ConvolutionKernel.h)
constexpr float kJincNormRadius = 0.96960938f;
constexpr float kJc0 = 0.999923599661866f, kJc1 = 0.014023570134078f, kJc2 = -2.969947516849635f,
                kJc3 = 0.891173008769047f, kJc4 = 2.326043034495162f, kJc5 = -1.270644932677047f;

struct SdcArgs {
    int D;
    int mos[3];
    float half_mos_pad[3];   // (mos + pad) / 2
    float hp;                // pad / 2
    float radius;
    int64_t M;
};

__device__ __forceinline__ float jinc_weight(const float *ad, int D, float R) {
    for (int d = 0; d < D; d++)
        if (ad[d] > R) return 0.f;
    float r = 0.f;
    for (int d = 0; d < D; d++) r += ad[d] * ad[d];
    r = sqrtf(r);
    r /= R;
    if (r >= kJincNormRadius) return 0.f;
    // the reference's sum c0 + c1 r + ... + c5 r^5 in its order, the powers
    // formed by products (within a few ulp of pow(r, k))
    const float r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r;
    float v = kJc0 + kJc1 * r + kJc2 * r2 + kJc3 * r3 + kJc4 * r4 + kJc5 * r5;
    return v < 0.f ? 0.f : v;
}

__device__ __forceinline__ int wrap_cell(int c, int m) { return c < 0 ? c + m : (c >= m ? c - m : c); }

// Visits this lane's share of the footprint cells of sample j (tap t =
// lane, lane + 32, ... in z, y, x order), calling f(cell_index, weight).
template <class F>
__device__ __forceinline__ void for_footprint_lane(const SdcArgs &a, const float *traj, int64_t j, int lane,
                                                   F &&f) {
    float s[3] = {0.f, 0.f, 0.f};
    int lo[3] = {0, 0, 0}, n[3] = {1, 1, 1};
    for (int d = 0; d < a.D; d++) {
        s[d] = fmaf(traj[j * a.D + d], (float)a.mos[d], a.half_mos_pad[d]) - a.hp;
        lo[d] = (int)ceilf(s[d] - a.radius);
        const int hi = (int)floorf(s[d] + a.radius);
        n[d] = hi >= lo[d] ? hi - lo[d] + 1 : 0;
    }
    const int taps = n[0] * n[1] * n[2];
    if (lane >= taps) return;
    // tap coordinates of t, stepped by 32 taps per round without divisions
    int tx = lane % n[0], ty = (lane / n[0]) % n[1], tz = lane / (n[0] * n[1]);
    for (int t = lane; t < taps; t += 32) {
        const int c[3] = {lo[0] + tx, lo[1] + ty, lo[2] + tz};
        float ad[3];
        for (int d = 0; d < a.D; d++) ad[d] = fabsf(s[d] - (float)c[d]);
        const float w = jinc_weight(ad, a.D, a.radius);
        if (isfinite(w) && w != 0.f) {
            int64_t idx = 0;
            for (int d = a.D - 1; d >= 0; d--) idx = idx * a.mos[d] + wrap_cell(c[d], a.mos[d]);
            f(idx, w);
        }
        tx += 32;
        while (tx >= n[0]) {
            tx -= n[0];
            if (++ty == n[1]) {
                ty = 0;
                ++tz;
            }
        }
    }
}

__global__ void k_sdc_grid(SdcArgs a, const float *__restrict__ traj, const float *__restrict__ w,
                           float *__restrict__ grid) {
    const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= a.M) return;
    const float v = w[j];
    for_footprint_lane(a, traj, j, threadIdx.x & 31, [&](int64_t idx, float wt) { atomicAdd(&grid[idx], wt * v); });
}

__global__ void k_sdc_degrid_update(SdcArgs a, const float *__restrict__ traj, const float *__restrict__ grid,
                                    float *__restrict__ w) {
    const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= a.M) return;   // whole warps leave together (blockDim is a multiple of 32)
    const int lane = threadIdx.x & 31;
    float t = 0.f;
    for_footprint_lane(a, traj, j, lane, [&](int64_t idx, float wt) { t += wt * grid[idx]; });
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) w[j] = t == 0.f ? 0.f : w[j] / t;
}

// Scratch kept per device between calls; the mutex is held for a whole call.
struct SdcScratch {
    std::mutex mu;
    DevBuf<unsigned int> bad;
    DevBuf<float> grid;
};

__global__ void k_fill(float *p, int64_t n, float v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_traj_range(const float *traj, int64_t n, unsigned int *bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float v = traj[i];
        if (!(v >= -0.5f && v <= 0.5f)) atomicOr(bad, 1u);
    }
}

}  // namespace

void sdc_estimate_dcw(int D, const uint64_t *N, float os_factor, int iterations, float kernel_width,
                      const float *traj, int64_t M, const float *initial, float *dcw, cudaStream_t st) {
    if (D < 1 || D > 3 || !N || !traj || !dcw || M <= 0 || iterations < 0)
        fail(GB_ERR_INVALID_ARGUMENT, "invalid density estimation arguments");
    if (!(os_factor >= 1.f) || !(kernel_width > 0.f)) fail(GB_ERR_INVALID_ARGUMENT, "invalid oversampling or width");
    SdcArgs a{};
    a.D = D;
    a.M = M;
    a.radius = kJincNormRadius * kernel_width;
    if (2.f * a.radius < 1.8f) fail(GB_ERR_INVALID_ARGUMENT, "Kernel width must be equal to or larger than 1.8.");
    const int pad = 2 * (int)std::ceil(a.radius);
    a.hp = (float)(pad / 2);
    int64_t G = 1;
    for (int d = 0; d < 3; d++) a.mos[d] = 1;
    for (int d = 0; d < D; d++) {
        if (N[d] == 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid matrix size");
        // vector_td<size_t>(vector_td<REAL>(N) * os), rounded up to a multiple of 32
        size_t m = (size_t)((float)N[d] * os_factor);
        m = ((m + 31) / 32) * 32;
        if (m > (1u << 20)) fail(GB_ERR_INVALID_ARGUMENT, "matrix size too large");
        a.mos[d] = (int)m;
        a.half_mos_pad[d] = (float)((m + pad) >> 1);
        G *= (int64_t)m;
    }
    const unsigned int tb = 256;
    const unsigned int sb = (unsigned int)((M + tb - 1) / tb);
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    SdcScratch &sc = device_scratch<SdcScratch>(dev);
    std::lock_guard<std::mutex> lock(sc.mu);
    {
        sc.bad.ensure(1);
        GB_CUDA(cudaMemsetAsync(sc.bad.get(), 0, sizeof(unsigned int), st));
        const int64_t nt = M * D;
        k_traj_range<<<(unsigned int)((nt + tb - 1) / tb), tb, 0, st>>>(traj, nt, sc.bad.get()); note_launch();
        unsigned int hb = 0;
        GB_CUDA(cudaMemcpyAsync(&hb, sc.bad.get(), sizeof(hb), cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaStreamSynchronize(st));
        if (hb) fail(GB_ERR_TRAJECTORY_RANGE, "trajectory out of range [-1/2, 1/2]");
    }
    if (initial) {
        if (initial != dcw) GB_CUDA(cudaMemcpyAsync(dcw, initial, M * sizeof(float), cudaMemcpyDeviceToDevice, st));
    } else {
        k_fill<<<sb, tb, 0, st>>>(dcw, M, 1.f); note_launch();
    }
    DevBuf<float> &grid = sc.grid;
    grid.ensure((size_t)G);
    // one warp per sample
    const unsigned int wb = (unsigned int)((M + (tb / 32) - 1) / (tb / 32));
    for (int it = 0; it < iterations; it++) {
        GB_CUDA(cudaMemsetAsync(grid.get(), 0, (size_t)G * sizeof(float), st));
        k_sdc_grid<<<wb, tb, 0, st>>>(a, traj, dcw, grid.get()); note_launch();
        k_sdc_degrid_update<<<wb, tb, 0, st>>>(a, traj, grid.get(), dcw); note_launch();
    }
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaStreamSynchronize(st));   // the grid is free for the next call on return
}

}  // namespace gb
