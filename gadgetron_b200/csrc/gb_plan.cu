// Plan creation, trajectory preprocessing (scaling, tile binning, sorting),
// deapodization tables and the cuFFT plan cache.
//
// Reference behaviour restated here:
//   - size/width checks: toolboxes/nfft/gpu/cuGriddingConvolution.cu:56-85
//   - trajectory range check and scaling k*mos + (mos+pad)/2:
//     toolboxes/nfft/gpu/cuGriddingConvolution.cu:128-172,
//     toolboxes/nfft/gpu/ConvolverNC2C_standard.cuh:25-39
//   - deapodization filter = 1 / (unscaled centred FFT of the kernel sampled
//     around mos/2): toolboxes/nfft/gpu/cuNFFT.cu:136-202.  The kernel is
//     separable, so the transform is the product of 1D transforms; each is
//     evaluated here in double on the host from the same float kernel values.
//
// What is new: instead of the reference's sort of (cell, sample) pairs
// (M * W^D keys, ConvolverNC2C_standard.cuh:162-190 and
// cuGriddingConvolution.cu:361-422) samples are binned by tile: one key per
// sample for its home tile, plus one (tile, sample) pair per tile touched
// (at most 2^D per sample) for the gridding lists.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "gb_internal.cuh"

namespace gb {

NufftPlan::~NufftPlan() {
    for (auto &kv : fft_plans) cufftDestroy(kv.second);
    for (auto &kv : fft_plans_om) cufftDestroy(kv.second);
    for (auto &g : prep_graph)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (h_stage) cudaFreeHost(h_stage);
    if (upload_done) {
        cudaEventSynchronize(upload_done);
        cudaEventDestroy(upload_done);
    }
    if (h_upload) cudaFreeHost(h_upload);
}

// Pinned staging for host -> device uploads of preprocess: waits until the
// previous uploads from it have been read, then returns room for `bytes`.
static unsigned char *upload_room(NufftPlan &p, size_t bytes) {
    if (p.upload_done) GB_CUDA(cudaEventSynchronize(p.upload_done));
    if (bytes > p.h_upload_n) {
        if (p.h_upload) GB_CUDA(cudaFreeHost(p.h_upload));
        p.h_upload = nullptr;
        p.h_upload_n = 0;
        GB_CUDA(cudaMallocHost((void **)&p.h_upload, bytes));
        p.h_upload_n = bytes;
    }
    return p.h_upload;
}

static void upload_issued(NufftPlan &p, cudaStream_t st) {
    if (!p.upload_done) GB_CUDA(cudaEventCreateWithFlags(&p.upload_done, cudaEventDisableTiming));
    GB_CUDA(cudaEventRecord(p.upload_done, st));
}

// Pinned host words of the plan (grown, never shrunk).
static uint32_t *stage_words(NufftPlan &p, size_t n) {
    if (n > p.h_stage_n) {
        if (p.h_stage) GB_CUDA(cudaFreeHost(p.h_stage));
        p.h_stage = nullptr;
        p.h_stage_n = 0;
        GB_CUDA(cudaMallocHost((void **)&p.h_stage, n * sizeof(uint32_t)));
        p.h_stage_n = n;
    }
    return p.h_stage;
}

static uint64_t mix_key(uint64_t h, uint64_t v) {
    for (int b = 0; b < 8; b++) {
        h ^= (v >> (8 * b)) & 0xffu;
        h *= 1099511628211ull;
    }
    return h;
}

// Runs a segment of device work on `st`: eagerly the first time a key is
// seen, recorded into a graph (on a private stream) and launched the second
// time, replayed from the recorded graph afterwards.  `work` must not
// allocate when its key repeats (the key covers every buffer it uses).
template <class Work>
static void run_prep_segment(NufftPlan::PrepGraph &g, uint64_t key, cudaStream_t st, Work &&work) {
    if (g.exec && g.key == key) {
        GB_CUDA(cudaGraphLaunch(g.exec, st));
        note_launch(g.kernels);
        return;
    }
    if (g.seen != key) {
        work(st);
        g.seen = key;
        return;
    }
    cudaStream_t cs;
    GB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    const uint64_t before = launch_count();
    GB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    try {
        work(cs);
    } catch (...) {
        cudaStreamEndCapture(cs, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        throw;
    }
    const cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    const uint64_t kernels = launch_count() - before;
    note_launch(0 - kernels);   // recorded, not launched
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    cudaError_t ei = ec;
    if (ec == cudaSuccess) ei = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    GB_CUDA(ei);
    g.key = key;
    g.kernels = kernels;
    GB_CUDA(cudaGraphLaunch(g.exec, st));
    note_launch(kernels);
}

static double host_kb1(float delta, const NufftPlan &p, int d) {
    // Same float arithmetic as the device helper (host: no contraction).
    const KParams &k = p.kp;
    if (delta > k.radius) return 0.0;
    float _tmp = 2.0f * delta * k.one_over_W;
    float tmp = _tmp * _tmp;
    float arg = k.beta[d] * std::sqrt(1.0f - tmp);
    float bessi = bessi0f_ref(arg);
    float w = k.mos_f[d] * bessi * k.one_over_W;
    return std::isfinite(w) ? (double)w : 0.0;
}

void plan_init(NufftPlan &p, int D, const uint64_t *N, const uint64_t *mos, float W,
               uint32_t flags) {
    if (D < 1 || D > kMaxD) fail(GB_ERR_INVALID_ARGUMENT, "D must be 1, 2 or 3");
    if (!N || !mos) fail(GB_ERR_INVALID_ARGUMENT, "NULL matrix size");
    if (!(W >= 1.8f)) fail(GB_ERR_INVALID_ARGUMENT, "Kernel width must be equal to or larger than 1.8.");
    if (W > 7.0f) fail(GB_ERR_INVALID_ARGUMENT, "Kernel width above 7 is not supported");
    for (int d = 0; d < D; d++) {
        if (N[d] == 0 || mos[d] == 0 || N[d] % 32 || mos[d] % 32)
            fail(GB_ERR_INVALID_ARGUMENT, "Matrix size must be a multiple of 32.");
        if (mos[d] < N[d])
            fail(GB_ERR_INVALID_ARGUMENT, "Oversampled matrix size must be greater than or equal to matrix size.");
        if (mos[d] > (1u << 20)) fail(GB_ERR_INVALID_ARGUMENT, "matrix size too large");
    }
    GB_CUDA(cudaGetDevice(&p.device));
    p.D = D;
    p.W = W;
    p.flags = flags;
    KParams &k = p.kp;
    std::memset(&k, 0, sizeof(k));
    k.D = D;
    k.radius = W / 2.0f;
    k.one_over_W = 1.0f / W;
    k.hw = (int)std::ceil(k.radius);
    k.G = 1;
    k.NN = 1;
    for (int d = 0; d < kMaxD; d++) {
        p.N[d] = d < D ? (int64_t)N[d] : 1;
        p.mos[d] = d < D ? (int64_t)mos[d] : 1;
        k.mos[d] = (int)p.mos[d];
        k.N[d] = (int)p.N[d];
        k.mos_f[d] = (float)p.mos[d];
        k.G *= p.mos[d];
        k.NN *= p.N[d];
        if (d < D) {
            // beta per dimension in float (ConvolutionKernel.hpp:286-303), with
            // os_factor = mos/N as the (N, mos, W) constructor computes it.
            float os = (float)mos[d] / (float)N[d];
            float w2 = W * W, os2 = os * os, h = os - 0.5f;
            float arg = w2 / os2 * (h * h) - 0.8f;
            k.beta[d] = (float)M_PI * std::sqrt(arg);
        }
    }
    if (k.G > (int64_t)1 << 31) fail(GB_ERR_INVALID_ARGUMENT, "oversampled grid exceeds 2^31 cells");

    // Default tiling: 2D 16x16, 3D 8x8x8, 1D 256; coil group 8.
    Tiling &t = p.tiling;
    if (D == 1) { t.tile[0] = 256; t.tile[1] = 1; t.tile[2] = 1; }
    if (D == 2) { t.tile[0] = 16; t.tile[1] = 16; t.tile[2] = 1; }
    if (D == 3) { t.tile[0] = 8; t.tile[1] = 8; t.tile[2] = 8; }
    for (int d = 0; d < D; d++)
        while (t.tile[d] > k.mos[d]) t.tile[d] >>= 1;
    t.cg = 8;
    for (int d = 0; d < kMaxD; d++) {
        k.tile[d] = d < D ? t.tile[d] : 1;
        k.ntiles[d] = d < D ? k.mos[d] / k.tile[d] : 1;
    }
    k.ntiles_total = k.ntiles[0] * k.ntiles[1] * k.ntiles[2];

    // Deapodization tables.  psi_d(g) = sum_u phi_d(|u|) cos(2 pi (g - mos/2) u / mos)
    // is the 1D unscaled centred transform of the kernel sampled at cells
    // c = mos/2 + u (exactly what cuNFFT.cu:136-202 computes, per dimension).
    p.maxN = 0;
    p.maxmos = 0;
    for (int d = 0; d < D; d++) {
        p.maxN = std::max(p.maxN, (int)p.N[d]);
        p.maxmos = std::max(p.maxmos, (int)p.mos[d]);
    }
    std::vector<float> h_img((size_t)D * p.maxN, 0.f), h_os((size_t)D * p.maxmos, 0.f);
    for (int d = 0; d < D; d++) {
        const int m = (int)p.mos[d];
        std::vector<double> phi;
        std::vector<int> us;
        for (int c = 0; c < m; c++) {
            float delta = std::fabs(0.5f * k.mos_f[d] - (float)c);
            double v = host_kb1(delta, p, d);
            if (v != 0.0) {
                phi.push_back(v);
                us.push_back(c - m / 2);
            }
        }
        const int off = (int)((p.mos[d] - p.N[d]) >> 1);
        for (int g = 0; g < m; g++) {
            double s = 0.0;
            for (size_t i = 0; i < phi.size(); i++)
                s += phi[i] * std::cos(2.0 * M_PI * (double)(g - m / 2) * (double)us[i] / (double)m);
            float inv = (float)(1.0 / s);
            h_os[(size_t)d * p.maxmos + g] = inv;
            int n = g - off;
            if (n >= 0 && n < (int)p.N[d]) h_img[(size_t)d * p.maxN + n] = inv;
        }
    }
    p.deap_img.ensure(h_img.size());
    p.deap_os.ensure(h_os.size());
    GB_CUDA(cudaMemcpy(p.deap_img.get(), h_img.data(), h_img.size() * sizeof(float), cudaMemcpyHostToDevice));
    GB_CUDA(cudaMemcpy(p.deap_os.get(), h_os.data(), h_os.size() * sizeof(float), cudaMemcpyHostToDevice));
}

// ------------------------------------------------------------ kernels ----

__device__ __forceinline__ int floor_div(int a, int b) {
    int q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

__device__ __forceinline__ uint32_t frame_of(const int64_t *off, uint32_t F, int64_t j) {
    uint32_t lo = 0, hi = F;   // find f with off[f] <= j < off[f+1]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= j) lo = mid; else hi = mid;
    }
    return lo;
}

// Scale the trajectory, check its range, and compute each sample's home key.
__global__ void k_scale_bin(KParams k, const float *__restrict__ traj, int64_t M,
                            const int64_t *__restrict__ frame_off, uint32_t F,
                            float *__restrict__ pos, uint32_t *__restrict__ key,
                            uint32_t *__restrict__ idx, int *__restrict__ range_err) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    int tcoord[kMaxD] = {0, 0, 0};
    bool bad = false;
    for (int d = 0; d < k.D; d++) {
        float kv = traj[j * k.D + d];
        if (!(kv >= -0.5f && kv <= 0.5f)) bad = true;
        // s = k*mos + (mos+pad)/2, the reference's trajectory_scale (evaluated
        // on the device there, where the multiply-add is contracted).
        float bias = (float)((k.mos[d] + 2 * k.hw) >> 1);
        float s = fmaf(kv, k.mos_f[d], bias);
        pos[(int64_t)d * M + j] = s;
        float sp = s - (float)k.hw;
        int c0 = (int)floorf(sp);
        int t = floor_div(c0, k.tile[d]);
        tcoord[d] = wrapmod(t, k.ntiles[d]);
    }
    if (bad) {
        atomicOr(range_err, 1);
        for (int d = 0; d < k.D; d++) tcoord[d] = 0;
    }
    uint32_t f = frame_of(frame_off, F, j);
    uint32_t tile = (uint32_t)((tcoord[2] * k.ntiles[1] + tcoord[1]) * k.ntiles[0] + tcoord[0]);
    key[j] = f * (uint32_t)k.ntiles_total + tile;
    idx[j] = (uint32_t)j;
}

__global__ void k_gather_pos(int D, int64_t M, const float *__restrict__ pos,
                             const uint32_t *__restrict__ perm, float *__restrict__ pos_sorted) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    uint32_t j = perm[i];
    for (int d = 0; d < D; d++) pos_sorted[(int64_t)d * M + i] = pos[(int64_t)d * M + j];
}

// Run offsets of a sorted key array: off[k] = first index whose key is >= k,
// off[nkeys] = n (no atomics: every thread fills the offsets between the key
// before it and its own).
__global__ void k_sorted_offsets(const uint32_t *__restrict__ keys, int64_t n, uint32_t nkeys,
                                 uint32_t *__restrict__ off) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    const int64_t prev = (i == 0) ? -1 : (int64_t)keys[i - 1];
    const int64_t cur = (i == n) ? (int64_t)nkeys : (int64_t)keys[i];
    for (int64_t k = prev + 1; k <= cur; k++) off[k] = (uint32_t)i;
}

// Tiles touched by the gridding footprint of sorted sample i (NC2C taps
// [ceil(s - W/2), floor(s + W/2)] on the padded grid, folded by -pad/2 and
// wrapped; ConvolverNC2C_standard.cuh:41-60,81-129 and :358-477).
__device__ __forceinline__ int touched_tiles(const KParams &k, const float *s, int tl[kMaxD][3],
                                             int nt[kMaxD]) {
    int total = 1;
    for (int d = 0; d < kMaxD; d++) {
        if (d >= k.D) { tl[d][0] = 0; nt[d] = 1; continue; }
        int lo = (int)ceilf(s[d] - k.radius) - k.hw;
        int hi = (int)floorf(s[d] + k.radius) - k.hw;
        int t0 = floor_div(lo, k.tile[d]);
        int t1 = floor_div(hi, k.tile[d]);
        int n = 0;
        for (int t = t0; t <= t1 && n < 3; t++) {
            int w = wrapmod(t, k.ntiles[d]);
            bool dup = false;
            for (int q = 0; q < n; q++) dup |= (tl[d][q] == w);
            if (!dup) tl[d][n++] = w;
        }
        nt[d] = n;
        total *= n;
    }
    return total;
}

// Per sorted sample and dimension, the 1D kernel weights of its taps
// t = 0..kWMax-1 at padded-grid cells ceil(s - W/2) + t (zero beyond the
// footprint): the values the convolution kernels would compute from the
// position, evaluated once per trajectory.
__global__ void k_weight_table(KParams k, int64_t M, const float *__restrict__ pos_sorted,
                               float4 *__restrict__ wtab) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * k.D) return;
    const int64_t j = e / k.D;
    const int d = (int)(e - j * k.D);
    const float s = pos_sorted[(int64_t)d * M + j];
    const int lo = (int)ceilf(s - k.radius);
    const int n = (int)floorf(s + k.radius) - lo + 1;
    float w[kWMax];
#pragma unroll
    for (int t = 0; t < kWMax; t++)
        w[t] = t < n ? kb_weight_1d(fabsf(s - (float)(lo + t)), k.mos_f[d], k.one_over_W, k.beta[d], k.radius) : 0.f;
    wtab[2 * e] = make_float4(w[0], w[1], w[2], w[3]);
    wtab[2 * e + 1] = make_float4(w[4], w[5], w[6], w[7]);
}

__global__ void k_count_pairs(KParams k, int64_t M, const float *__restrict__ pos_sorted,
                              uint32_t *__restrict__ cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    float s[kMaxD] = {0.f, 0.f, 0.f};
    for (int d = 0; d < k.D; d++) s[d] = pos_sorted[(int64_t)d * M + i];
    int tl[kMaxD][3], nt[kMaxD];
    cnt[i] = (uint32_t)touched_tiles(k, s, tl, nt);
}

__global__ void k_write_pairs(KParams k, int64_t M, const float *__restrict__ pos_sorted,
                              const uint32_t *__restrict__ sorted_home_key,
                              const uint32_t *__restrict__ pair_off,
                              uint32_t *__restrict__ pkey, uint32_t *__restrict__ pval) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    float s[kMaxD] = {0.f, 0.f, 0.f};
    for (int d = 0; d < k.D; d++) s[d] = pos_sorted[(int64_t)d * M + i];
    int tl[kMaxD][3], nt[kMaxD];
    touched_tiles(k, s, tl, nt);
    uint32_t frame = sorted_home_key[i] / (uint32_t)k.ntiles_total;
    uint32_t o = pair_off[i];
    for (int a = 0; a < nt[2]; a++)
        for (int b = 0; b < nt[1]; b++)
            for (int c = 0; c < nt[0]; c++) {
                uint32_t tile = (uint32_t)((tl[2][a] * k.ntiles[1] + tl[1][b]) * k.ntiles[0] + tl[0][c]);
                pkey[o] = frame * (uint32_t)k.ntiles_total + tile;
                pval[o] = (uint32_t)i;
                o++;
            }
}

// Pair rows for the row-variant gridding kernel: one thread per (pair,
// dimension) lays the sample's tap weights (from the weight table, unsigned)
// over the tile's extent in that dimension -- tap t at tile-local cell
// (ceil(s - W/2) + t - pad/2 - tile origin) mod mos when that falls inside the
// tile, zero elsewhere -- and records the tile-local footprint range.
__global__ void k_pair_rows(KParams k, int64_t M, int64_t npairs, const float *__restrict__ pos_sorted,
                            const float *__restrict__ wtab, const uint32_t *__restrict__ pair_key,
                            const uint32_t *__restrict__ pair_sample, float *__restrict__ rows, int row_floats,
                            int row_weights) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npairs * k.D) return;
    const int64_t q = e / k.D;
    const int d = (int)(e - q * k.D);
    const uint32_t si = pair_sample[q];
    const uint32_t tile = pair_key[q] % (uint32_t)k.ntiles_total;
    const int tc = d == 0 ? (int)(tile % k.ntiles[0])
                          : (d == 1 ? (int)((tile / k.ntiles[0]) % k.ntiles[1])
                                    : (int)(tile / (k.ntiles[0] * k.ntiles[1])));
    const int Td = k.tile[d];
    const int org = tc * Td;
    const float sp = pos_sorted[(int64_t)d * M + si];
    const int lo = (int)ceilf(sp - k.radius);
    const int n = min((int)floorf(sp + k.radius) - lo + 1, kWMax);
    int a0 = lo - k.hw - org;   // tile-local footprint start, mod mos
    a0 = a0 < 0 ? a0 + k.mos[d] : (a0 >= k.mos[d] ? a0 - k.mos[d] : a0);
    float *row = rows + q * row_floats;
    float *wr = row + (d == 0 ? 0 : (d == 1 ? k.tile[0] : k.tile[0] + k.tile[1]));
    const float *taps = wtab + ((int64_t)si * k.D + d) * kWMax;
    for (int c = 0; c < Td; c++) {
        int t = c - a0;
        if (t < 0) t += k.mos[d];
        wr[c] = t < n ? taps[t] : 0.f;
    }
    if (d == 0)
        for (int c = k.tile[0] + k.tile[1] + (k.D == 3 ? k.tile[2] : 0); c < row_weights; c++) row[c] = 0.f;
    int rlo, rhi;
    if (k.ntiles[d] == 1) {   // the footprint may wrap inside the tile
        rlo = 0;
        rhi = Td - 1;
    } else {
        const int st = (a0 < Td) ? a0 : a0 - k.mos[d];
        rlo = max(st, 0);
        rhi = min(st + n - 1, Td - 1);
    }
    reinterpret_cast<uint32_t *>(row + row_weights)[d] = (uint32_t)rlo | ((uint32_t)rhi << 16);
    if (d == 0 && k.D == 2) reinterpret_cast<uint32_t *>(row + row_weights)[2] = 0u;
}

static int bits_for(uint64_t n) {
    int b = 1;
    while ((1ull << b) < n) b++;
    return b;
}

void plan_preprocess(NufftPlan &p, const float *traj, uint64_t Mtot, uint32_t F,
                     const uint64_t *frame_offsets, gb_prep_mode mode, cudaStream_t st) {
    if (!traj) fail(GB_ERR_INVALID_ARGUMENT, "NULL trajectory");
    if (Mtot == 0 || F == 0) fail(GB_ERR_INVALID_ARGUMENT, "empty trajectory");
    if (Mtot >= (1ull << 31)) fail(GB_ERR_INVALID_ARGUMENT, "too many samples (>= 2^31)");
    if ((uint64_t)F * (uint64_t)p.kp.ntiles_total >= (1ull << 31))
        fail(GB_ERR_INVALID_ARGUMENT, "too many frames for the tile grid");
    std::vector<int64_t> off(F + 1);
    if (frame_offsets) {
        for (uint32_t f = 0; f <= F; f++) off[f] = (int64_t)frame_offsets[f];
        if (off[0] != 0 || off[F] != (int64_t)Mtot)
            fail(GB_ERR_INVALID_ARGUMENT, "frame offsets must start at 0 and end at the sample count");
        for (uint32_t f = 0; f < F; f++)
            if (off[f + 1] < off[f]) fail(GB_ERR_INVALID_ARGUMENT, "frame offsets must be non-decreasing");
    } else {
        if (Mtot % F) fail(GB_ERR_INVALID_ARGUMENT, "sample count is not a multiple of the frame count");
        for (uint32_t f = 0; f <= F; f++) off[f] = (int64_t)(Mtot / F) * f;
    }
    p.prepped = false;
    p.generation++;
    const KParams &k = p.kp;
    const int64_t M = (int64_t)Mtot;
    const int D = p.D;
    const uint32_t nkeys = F * (uint32_t)k.ntiles_total;

    // Keep the trajectory (re-binning for the autotuner needs it).
    if (traj != p.traj_copy.get()) {
        p.traj_copy.ensure((size_t)D * M);
        GB_CUDA(cudaMemcpyAsync(p.traj_copy.get(), traj, (size_t)D * M * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    DevBuf<int64_t> &d_off = p.pp_off;
    d_off.ensure(F + 1);
    {
        unsigned char *up = upload_room(p, (F + 1) * sizeof(int64_t));
        std::memcpy(up, off.data(), (F + 1) * sizeof(int64_t));
        GB_CUDA(cudaMemcpyAsync(d_off.get(), up, (F + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        upload_issued(p, st);
    }
    DevBuf<float> &pos = p.pp_pos;
    pos.ensure((size_t)D * M);
    DevBuf<uint32_t> &key = p.pp_key, &idx = p.pp_idx, &key_sorted = p.pp_key_sorted;
    key.ensure(M);
    idx.ensure(M);
    key_sorted.ensure(M);
    DevBuf<int> &err = p.pp_err;
    err.ensure(1);
    p.perm.ensure(M);
    p.pos_sorted.ensure((size_t)D * M);
    p.wtab.ensure((size_t)M * D * kWMax);
    p.home_off.ensure(nkeys + 1);
    DevBuf<uint32_t> &pcnt = p.pp_pcnt, &poff = p.pp_poff;
    pcnt.ensure(M + 1);
    poff.ensure(M + 1);
    const int TB = 256;
    uint64_t kp_hash = 1469598103934665603ull;
    {
        uint64_t w[(sizeof(KParams) + 7) / 8] = {};
        std::memcpy(w, &k, sizeof(KParams));
        for (uint64_t v : w) kp_hash = mix_key(kp_hash, v);
    }

    // Segment A: scaling and range check, home keys, stable sort of the
    // samples by (frame, home tile), sorted positions, weight table, home
    // ranges, pair counts and their scan.  Until the range flag is read
    // back with the pair count, out-of-range samples sit in tile 0 and every
    // kernel in between stays in bounds for any position value.
    uint64_t key_a = kp_hash;
    for (uint64_t v : {(uint64_t)(uintptr_t)traj, (uint64_t)M, (uint64_t)F, (uint64_t)nkeys,
                       (uint64_t)(uintptr_t)d_off.get(), (uint64_t)(uintptr_t)pos.get(), (uint64_t)(uintptr_t)key.get(),
                       (uint64_t)(uintptr_t)idx.get(), (uint64_t)(uintptr_t)key_sorted.get(),
                       (uint64_t)(uintptr_t)err.get(), (uint64_t)(uintptr_t)p.perm.get(),
                       (uint64_t)(uintptr_t)p.pos_sorted.get(), (uint64_t)(uintptr_t)p.wtab.get(),
                       (uint64_t)(uintptr_t)p.home_off.get(), (uint64_t)(uintptr_t)pcnt.get(),
                       (uint64_t)(uintptr_t)poff.get(), (uint64_t)(uintptr_t)p.pp_sort.get(), (uint64_t)p.pp_sort.n})
        key_a = mix_key(key_a, v);
    run_prep_segment(p.prep_graph[0], key_a, st, [&](cudaStream_t s) {
        GB_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
        k_scale_bin<<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(k, traj, M, d_off.get(), F, pos.get(),
                                                                  key.get(), idx.get(), err.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        sort_pairs(key.get(), key_sorted.get(), idx.get(), p.perm.get(), M, bits_for(nkeys), p.pp_sort, s);
        k_gather_pos<<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(D, M, pos.get(), p.perm.get(),
                                                                   p.pos_sorted.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        k_weight_table<<<(unsigned)((M * D + TB - 1) / TB), TB, 0, s>>>(k, M, p.pos_sorted.get(),
                                                                        reinterpret_cast<float4 *>(p.wtab.get())); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        k_sorted_offsets<<<(unsigned)((M + TB) / TB), TB, 0, s>>>(key_sorted.get(), M, (uint32_t)nkeys,
                                                                 p.home_off.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        GB_CUDA(cudaMemsetAsync(pcnt.get() + M, 0, sizeof(uint32_t), s));
        k_count_pairs<<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(k, M, p.pos_sorted.get(), pcnt.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        exclusive_scan(pcnt.get(), poff.get(), M + 1, p.pp_sort, s);
    });
    uint32_t *hs = stage_words(p, 2);
    GB_CUDA(cudaMemcpyAsync(hs, poff.get() + M, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaMemcpyAsync(hs + 1, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    const uint32_t npairs = hs[0];
    if (hs[1]) fail(GB_ERR_TRAJECTORY_RANGE, "trajectory out of range [-1/2, 1/2]");
    p.total_pairs = npairs;

    // Segment B: the gridding pair lists -- (tile, sample) pairs written,
    // stably sorted by (frame, tile), their ranges, and the pair rows of the
    // row-variant gridding (2D/3D tiles up to 96 cells of extent sum).
    DevBuf<uint32_t> &pkey = p.pp_pkey, &pval = p.pp_pval, &pkey_sorted = p.pp_pkey_sorted;
    pkey.ensure(npairs);
    pval.ensure(npairs);
    pkey_sorted.ensure(npairs);
    p.grid_list.ensure(npairs);
    p.grid_off.ensure(nkeys + 1);
    const bool rows = D >= 2 && pair_row_weights(k) <= 96 && npairs > 0;
    const int rf = rows ? pair_row_floats(k) : 0;
    if (rows) p.pair_rows.ensure((size_t)npairs * rf);
    uint64_t key_b = kp_hash;
    for (uint64_t v : {(uint64_t)npairs, (uint64_t)M, (uint64_t)nkeys, (uint64_t)rf,
                       (uint64_t)(uintptr_t)p.pos_sorted.get(), (uint64_t)(uintptr_t)key_sorted.get(),
                       (uint64_t)(uintptr_t)poff.get(), (uint64_t)(uintptr_t)pkey.get(), (uint64_t)(uintptr_t)pval.get(),
                       (uint64_t)(uintptr_t)pkey_sorted.get(), (uint64_t)(uintptr_t)p.grid_list.get(),
                       (uint64_t)(uintptr_t)p.grid_off.get(), (uint64_t)(uintptr_t)p.wtab.get(),
                       (uint64_t)(uintptr_t)p.pair_rows.get(), (uint64_t)(uintptr_t)p.pp_sort.get(),
                       (uint64_t)p.pp_sort.n})
        key_b = mix_key(key_b, v);
    run_prep_segment(p.prep_graph[1], key_b, st, [&](cudaStream_t s) {
        k_write_pairs<<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(k, M, p.pos_sorted.get(), key_sorted.get(),
                                                                    poff.get(), pkey.get(), pval.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        sort_pairs(pkey.get(), pkey_sorted.get(), pval.get(), p.grid_list.get(), npairs, bits_for(nkeys), p.pp_sort, s);
        k_sorted_offsets<<<(unsigned)(((int64_t)npairs + TB) / TB), TB, 0, s>>>(pkey_sorted.get(), npairs,
                                                                               (uint32_t)nkeys, p.grid_off.get()); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        if (rows) {
            k_pair_rows<<<(unsigned)(((int64_t)npairs * D + TB - 1) / TB), TB, 0, s>>>(
                k, M, npairs, p.pos_sorted.get(), p.wtab.get(), pkey_sorted.get(), p.grid_list.get(), p.pair_rows.get(),
                rf, pair_row_weights(k)); ::gb::note_launch();
            GB_CUDA(cudaGetLastError());
        }
    });
    p.pair_row_stride = rf;
    if (p.err_flag.ensure(1)) GB_CUDA(cudaMemsetAsync(p.err_flag.get(), 0, sizeof(unsigned int), st));

    p.F = F;
    p.Mtot = M;
    p.frame_off = off;
    p.prepped_c2nc = (mode == GB_PREP_C2NC || mode == GB_PREP_ALL);
    p.prepped_nc2c = (mode == GB_PREP_NC2C || mode == GB_PREP_ALL);
    // Both structures are built regardless of mode (they are cheap); the mode
    // is recorded for the reference's precondition checks.
    p.prepped_c2nc = p.prepped_nc2c = true;
    p.prep_mode = mode;
    plan_build_work(p, st);
    fft_custom_prepare(p, st);
    p.prepped = true;
}

// Stable sort of work items by length, longest first (the same order as a
// std::stable_sort on that key): a counting sort when the lengths are small,
// as they are for tile lists -- this runs in every preprocess.
static void sort_items_by_length(std::vector<WorkItem> &v) {
    if (v.size() < 2) return;
    int maxlen = 0;
    for (const WorkItem &w : v) maxlen = std::max(maxlen, w.end - w.begin);
    if (maxlen > (1 << 16)) {
        std::stable_sort(v.begin(), v.end(), [](const WorkItem &a, const WorkItem &b) {
            return (a.end - a.begin) > (b.end - b.begin);
        });
        return;
    }
    std::vector<uint32_t> start((size_t)maxlen + 2, 0u);
    for (const WorkItem &w : v) start[(size_t)(maxlen - (w.end - w.begin)) + 1]++;
    for (size_t i = 1; i < start.size(); i++) start[i] += start[i - 1];
    std::vector<WorkItem> out(v.size());
    for (const WorkItem &w : v) out[start[(size_t)(maxlen - (w.end - w.begin))]++] = w;
    v.swap(out);
}

// Host-side work lists: degridding chunks of home samples, gridding tiles
// (heavy tiles split into chunks reduced by the last CTA).
void plan_build_work(NufftPlan &p, cudaStream_t st) {
    const KParams &k = p.kp;
    const uint32_t nkeys = p.F * (uint32_t)k.ntiles_total;
    uint32_t *hoff = stage_words(p, 2 * ((size_t)nkeys + 1));   // pinned: both readbacks, one synchronisation
    uint32_t *goff = hoff + nkeys + 1;
    GB_CUDA(cudaMemcpyAsync(hoff, p.home_off.get(), (nkeys + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaMemcpyAsync(goff, p.grid_off.get(), (nkeys + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    p.h_home_counts.resize(nkeys);
    for (uint32_t i = 0; i < nkeys; i++) p.h_home_counts[i] = hoff[i + 1] - hoff[i];

    // Degridding items: chunks of at most `deg_chunk` home samples.
    const int64_t M = p.Mtot;
    // (large enough that a tile is staged once or a few times; the region
    // copy is a large share of an item's work in 2D)
    int deg_chunk = (int)std::max<int64_t>(256, std::min<int64_t>(1024, M / (148 * 4) + 1));
    std::vector<WorkItem> deg;
    for (uint32_t key = 0; key < nkeys; key++) {
        uint32_t b = hoff[key], e = hoff[key + 1];
        for (uint32_t s = b; s < e; s += deg_chunk) {
            WorkItem w{};
            w.ft = (int)key;
            w.begin = (int)s;
            w.end = (int)std::min<uint32_t>(e, s + deg_chunk);
            w.split = -1;
            deg.push_back(w);
        }
    }
    sort_items_by_length(deg);

    // Gridding items.
    int64_t total = goff[nkeys];
    int split_len = p.tiling.split_len;
    if (split_len <= 0) {
        int64_t avg = total / std::max<uint32_t>(1, nkeys);
        split_len = (int)std::max<int64_t>(256, 2 * avg);
    }
    std::vector<WorkItem> heavy, light;
    std::vector<SplitInfo> splits;
    int slots = 0;
    for (uint32_t key = 0; key < nkeys; key++) {
        uint32_t b = goff[key], e = goff[key + 1];
        uint32_t len = e - b;
        if ((int)len <= split_len) {
            WorkItem w{};
            w.ft = (int)key;
            w.begin = (int)b;
            w.end = (int)e;
            w.split = -1;
            light.push_back(w);
        } else {
            int nch = (int)((len + split_len - 1) / split_len);
            int per = (int)((len + nch - 1) / nch);
            SplitInfo si{slots, nch};
            int sid = (int)splits.size();
            splits.push_back(si);
            for (int c = 0; c < nch; c++) {
                WorkItem w{};
                w.ft = (int)key;
                w.begin = (int)(b + c * per);
                w.end = (int)std::min<uint32_t>(e, b + (c + 1) * per);
                w.split = sid;
                w.chunk = c;
                heavy.push_back(w);
            }
            slots += nch;
        }
    }
    sort_items_by_length(light);
    std::vector<WorkItem> grd(heavy);
    grd.insert(grd.end(), light.begin(), light.end());

    p.n_deg_items = (int)deg.size();
    p.deg_items.ensure(std::max<size_t>(1, deg.size()));
    p.n_grd_items = (int)grd.size();
    p.grd_items.ensure(std::max<size_t>(1, grd.size()));
    p.n_splits = (int)splits.size();
    p.n_slots = slots;
    p.splits.ensure(std::max<size_t>(1, splits.size()));
    // The three lists go up from pinned staging (asynchronous; the staging
    // is not rewritten before these copies have been read).
    const size_t bd = deg.size() * sizeof(WorkItem), bg = grd.size() * sizeof(WorkItem);
    const size_t bs = splits.size() * sizeof(SplitInfo);
    unsigned char *up = upload_room(p, bd + bg + bs);
    if (bd) std::memcpy(up, deg.data(), bd);
    if (bg) std::memcpy(up + bd, grd.data(), bg);
    if (bs) std::memcpy(up + bd + bg, splits.data(), bs);
    if (bd) GB_CUDA(cudaMemcpyAsync(p.deg_items.get(), up, bd, cudaMemcpyHostToDevice, st));
    if (bg) GB_CUDA(cudaMemcpyAsync(p.grd_items.get(), up + bd, bg, cudaMemcpyHostToDevice, st));
    if (bs) GB_CUDA(cudaMemcpyAsync(p.splits.get(), up + bd + bg, bs, cudaMemcpyHostToDevice, st));
    upload_issued(p, st);
    p.split_counter_groups = 0;   // (re)allocated by the gridding launcher
}

uint64_t plan_layout_signature(const NufftPlan &p, int nbf) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int b = 0; b < 8; b++) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    const void *ptrs[] = {p.pos_sorted.get(), p.wtab.get(), p.pair_rows.get(), p.perm.get(), p.grid_list.get(), p.grd_items.get(),
                          p.deg_items.get(), p.splits.get(), p.partials.get(), p.split_counters.get(), p.grid_queue.get(),
                          p.img_os.get(), p.kgrid.get(), p.samp_ws.get(), p.deap_img.get(), p.deap_os.get()};
    for (const void *q : ptrs) mix((uint64_t)(uintptr_t)q);
    const int64_t vals[] = {p.n_deg_items, p.n_grd_items, p.n_splits, p.n_slots, p.Mtot, (int64_t)p.F,
                            p.tiling.tile[0], p.tiling.tile[1], p.tiling.tile[2], p.tiling.cg, p.tiling.schedule,
                            p.split_counter_groups, (int64_t)p.split_counters.n, (int64_t)p.partials.n, nbf};
    for (int64_t v : vals) mix((uint64_t)v);
    auto it = p.fft_plans.find(nbf);
    mix(it == p.fft_plans.end() ? 0ull : (uint64_t)it->second);
    for (int pass = 0; pass < 3; pass++) {
        auto jt = p.fft_plans_om.find(std::make_pair(nbf, pass));
        mix(jt == p.fft_plans_om.end() ? 0ull : (uint64_t)jt->second);
    }
    return h;
}

// The tiling a new plan starts with: 16 x 16 (2D), 256 (1D), 8^3 (3D),
// shrunk to the grid for small grids; coil group 16.
void plan_default_tiling(NufftPlan &p) {
    int t[3] = {16, 16, 1};
    if (p.D == 1) { t[0] = 256; }
    if (p.D == 3) { t[0] = 8; t[1] = 8; t[2] = 8; }
    for (int d = 0; d < p.D; d++)
        if (t[d] > p.kp.mos[d]) t[d] = (int)p.kp.mos[d];
    plan_set_tiling(p, t, 16);
}

// Validates and installs a tiling (tile shape and coil group).
void plan_set_tiling(NufftPlan &p, const int *tile, int cg) {
    const KParams &k = p.kp;
    int t[kMaxD] = {1, 1, 1};
    for (int d = 0; d < p.D; d++) t[d] = tile[d];
    int cells = t[0] * t[1] * t[2];
    for (int d = 0; d < p.D; d++)
        if (t[d] <= 0 || k.mos[d] % t[d]) fail(GB_ERR_INVALID_ARGUMENT, "tile size must divide the oversampled size");
    if (p.D == 1) {
        if (t[0] % 32) fail(GB_ERR_INVALID_ARGUMENT, "1D tile must be a multiple of 32");
    } else if (t[0] % 8 || t[1] % 4) {
        fail(GB_ERR_INVALID_ARGUMENT, "tile x must be a multiple of 8 and y a multiple of 4");
    }
    if (cells > 4 * kThreads || (cells > kThreads && cells % kThreads) || (cells < kThreads && kThreads % cells))
        fail(GB_ERR_INVALID_ARGUMENT, "tile must hold a divisor of 256 cells, or 512 or 1024 cells");
    if (2 * k.hw + 1 > kWMax) fail(GB_ERR_INVALID_ARGUMENT, "kernel width too large");
    // A footprint of at most 2*hw+1 cells must span at most 3 tiles per
    // dimension (the binning records up to 3 tiles per dimension).
    for (int d = 0; d < p.D; d++)
        if (t[d] < 2 * k.hw && t[d] != k.mos[d])
            fail(GB_ERR_INVALID_ARGUMENT, "tile must be at least W cells wide in every dimension");
    if (cg != 1 && cg != 2 && cg != 4 && cg != 8 && cg != 16)
        fail(GB_ERR_INVALID_ARGUMENT, "coil group must be 1, 2, 4, 8 or 16");
    p.tiling.cg = cg;
    for (int d = 0; d < kMaxD; d++) {
        p.tiling.tile[d] = t[d];
        p.kp.tile[d] = t[d];
        p.kp.ntiles[d] = p.kp.mos[d] / t[d];
    }
    p.kp.ntiles_total = p.kp.ntiles[0] * p.kp.ntiles[1] * p.kp.ntiles[2];
}


cufftHandle plan_fft(NufftPlan &p, int batches, cudaStream_t st) {
    auto it = p.fft_plans.find(batches);
    cufftHandle h;
    if (it == p.fft_plans.end()) {
        int n[kMaxD];
        for (int d = 0; d < p.D; d++) n[d] = (int)p.mos[p.D - 1 - d];
        int dist = (int)p.kp.G;
        GB_CUFFT(cufftPlanMany(&h, p.D, n, n, 1, dist, n, 1, dist, CUFFT_C2C, batches));
        p.fft_plans[batches] = h;
    } else {
        h = it->second;
    }
    GB_CUFFT(cufftSetStream(h, st));
    return h;
}

int64_t fft_band_offset(const NufftPlan &p, int nbf) {
    const KParams &k = p.kp;
    if (p.D == 2) return (int64_t)((k.mos[1] - k.N[1]) / 2) * nbf * k.mos[0];
    return (int64_t)((k.mos[2] - k.N[2]) / 2) * nbf * k.mos[1] * k.mos[0];
}

cufftHandle plan_fft_om(NufftPlan &p, int nbf, FftPass pass, cudaStream_t st) {
    if (p.D < 2) fail(GB_ERR_INTERNAL, "outer-major FFT passes need D >= 2");
    const auto key = std::make_pair(nbf, (int)pass);
    auto it = p.fft_plans_om.find(key);
    cufftHandle h;
    if (it == p.fft_plans_om.end()) {
        const KParams &k = p.kp;
        if (pass == FFT_PASS_B) {
            // the outer dimension: stride = one outer step (all batches' inner planes)
            const int inner = p.D == 2 ? k.mos[0] : k.mos[1] * k.mos[0];
            int n[1] = {p.D == 2 ? k.mos[1] : k.mos[2]};
            const long long stride = (long long)nbf * inner;
            if (stride > INT32_MAX) fail(GB_ERR_INVALID_ARGUMENT, "k-space workspace too large for the FFT plan");
            GB_CUFFT(cufftPlanMany(&h, 1, n, n, (int)stride, 1, n, (int)stride, 1, CUFFT_C2C, nbf * inner));
        } else {
            const int outer = pass == FFT_PASS_A_BAND ? (p.D == 2 ? k.N[1] : k.N[2]) : (p.D == 2 ? k.mos[1] : k.mos[2]);
            if (p.D == 2) {
                int n[1] = {k.mos[0]};
                GB_CUFFT(cufftPlanMany(&h, 1, n, n, 1, k.mos[0], n, 1, k.mos[0], CUFFT_C2C, outer * nbf));
            } else {
                int n[2] = {k.mos[1], k.mos[0]};
                const int dist = k.mos[1] * k.mos[0];
                GB_CUFFT(cufftPlanMany(&h, 2, n, n, 1, dist, n, 1, dist, CUFFT_C2C, outer * nbf));
            }
        }
        p.fft_plans_om[key] = h;
    } else {
        h = it->second;
    }
    GB_CUFFT(cufftSetStream(h, st));
    return h;
}

}  // namespace gb
