// Gridding (NC2C), degridding (C2NC) and trajectory-gradient kernels.
//
// Reference kernels these replace:
//   NC2C  toolboxes/nfft/gpu/ConvolverNC2C_standard.cuh:229-355 (+ the wrap
//         pass :358-477 and the cell/sample pair sort of
//         toolboxes/nfft/gpu/cuGriddingConvolution.cu:361-422)
//   C2NC  toolboxes/nfft/gpu/ConvolverC2NC.cuh:78-122,228-307 (+ the coil-
//         fastest permute of cuGriddingConvolution.cu:329-334)
//
// Arithmetic kept identical to the reference: taps run over
// [ceil(s - W/2), floor(s + W/2)] per dimension, each tap's weight is the
// product over dimensions of the 1D Kaiser-Bessel value of |s - cell|
// (zero beyond W/2, non-finite weights dropped), and the periodic wrap maps a
// tap to (cell mod mos).  For NC2C s is the padded-grid coordinate and the
// cell is folded by -pad/2; for C2NC s - pad/2 is used directly
// (ConvolverC2NC.cuh:239-241).
//
// B200 design:
//   * gridding is output-driven per tile: a CTA owns a tile of the
//     oversampled grid, each thread owns CPT cells and accumulates a group of
//     CG coils in registers; a warp covers an 8x4 patch of cells so that a
//     sample footprint lights up a dense block of lanes.  Samples touching the
//     tile are staged 32 at a time in shared memory (positions -> separable
//     weights, values with the density weights folded in).  No atomics: the
//     result is bit-reproducible.  Tiles with long sample lists are split
//     over several CTAs whose partial tiles are summed in a fixed order by
//     the last CTA to finish.
//   * degridding stages the home tile plus a halo of pad/2 cells, coil
//     fastest, in shared memory; a warp serves one sample at a time with its
//     lanes over (coil, re/im), the separable weights are computed by 8 lanes
//     per dimension and broadcast by shuffles.
//   * the centring checkerboard of the centred FFT ((-1)^(sum of cell
//     coordinates), cuNDFFT.cu:6-36) is folded into the separable weights
//     (sign_fold), and the density weights are folded into the sample loads
//     (gridding) or stores (degridding).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

struct ConvArgs {
    KParams k;
    const float *pos;         // [D][Mtot] sorted positions
    const float *wtab;        // [Mtot][D][kWMax] tap weights of sorted samples
    const uint32_t *perm;     // sorted -> original
    const uint32_t *list;     // gridding list (sorted positions) or unused
    const WorkItem *items;
    int n_items;
    int64_t Mtot;
    int F;
    int nb;
    int layout;               // SampleLayout
    int il_stride;            // SORTED_IL: float2 per sample row (nb rounded up to even)
    const uint32_t *home_key; // sorted home keys (frame * ntiles_total + tile)
    const float *dcw;         // original order, may be null
    int dcw_pow;
    int sign_fold;
    int accumulate;
    // gridding split bookkeeping
    const SplitInfo *splits;
    float2 *partials;
    unsigned int *counters;
    int ncg;
    long long part_elems;     // float2 elements of one CTA's partial tile
    KLayout kl;               // k-space array layout
    const float *prows;       // gridding pair rows (row variant)
    int prow_floats;
    unsigned int *err;        // bounded-wait failure flag
    unsigned int *queue;      // persistent gridding: [0] next work unit, [1] CTAs finished
    int n_work;               // persistent gridding: work units (items x coil groups)
};

__device__ __forceinline__ float sign_of(int g) { return (g & 1) ? -1.f : 1.f; }

// --------------------------------------------------------------- NC2C -----

// Shared-memory stage of one chunk of kChunk samples for the gridding kernel.
template <int CG>
struct GridStage {
    float w[kChunk][3][kWMax];   // separable weights (checkerboard folded in)
    float2 v[kChunk][CG];        // sample values (density weights folded in)
    int a[kChunk][3];            // tile-local start of the footprint (wrapped)
    int n[kChunk][3];            // taps per dimension
    uint32_t mask[kChunk];       // warps whose cell patches the footprint overlaps
};

template <int CG, int CPT, bool COMP>
__global__ void __launch_bounds__(kThreads)
k_grid_nc2c(ConvArgs a, const float2 *__restrict__ samples, float2 *__restrict__ grid) {
    const KParams &k = a.k;
    const int item_idx = blockIdx.x;
    const int grp = blockIdx.y;
    const int b0 = grp * CG;
    const WorkItem it = a.items[item_idx];
    const int f = it.ft / k.ntiles_total;
    const int tile = it.ft - f * k.ntiles_total;
    const int tx = tile % k.ntiles[0];
    const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
    const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
    const int org[3] = {tx * k.tile[0], ty * k.tile[1], tz * k.tile[2]};

    __shared__ GridStage<CG> stage[2];
    __shared__ int s_last;

    // Cell ownership: warp patches of PX x PY cells.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int PX = (k.D == 1) ? 32 : 8;
    const int PY = (k.D == 1) ? 1 : 4;
    const int npx = k.tile[0] / PX, npy = k.tile[1] / PY;
    int lc[CPT][3];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        int q = warp + 8 * c;
        int qx = q % npx, qy = (q / npx) % npy, qz = q / (npx * npy);
        lc[c][0] = qx * PX + (lane % PX);
        lc[c][1] = qy * PY + (lane / PX);
        lc[c][2] = qz;
    }

    float acc[CPT][CG][2];
    float cmp[COMP ? CPT : 1][COMP ? CG : 1][2];
#pragma unroll
    for (int c = 0; c < CPT; c++)
#pragma unroll
        for (int q = 0; q < CG; q++) {
            acc[c][q][0] = acc[c][q][1] = 0.f;
            if (COMP) cmp[c][q][0] = cmp[c][q][1] = 0.f;
        }

    // Staging work per thread: weight entries (sample, dim, tap), value
    // entries (sample, coil) and, for threads < kChunk, one sample's
    // footprint and warp mask.  Raw global values are prefetched into
    // registers one chunk ahead so their latency overlaps the accumulation.
    constexpr int kWE = (kChunk * 3 * kWMax + kThreads - 1) / kThreads;
    constexpr int kVE = (kChunk * CG + kThreads - 1) / kThreads;
    float pw[kWE], pt[kWE];
    float2 pv[kVE];
    float pd[kVE];
    float ps[3];

    auto prefetch = [&](int base, int cnt) {
#pragma unroll
        for (int q = 0; q < kWE; q++) {
            const int e = threadIdx.x + q * kThreads;
            const int i = e / (3 * kWMax), d = (e / kWMax) % 3;
            pw[q] = 0.f;
            pt[q] = 0.f;
            if (e < kChunk * 3 * kWMax && i < cnt && d < k.D) {
                const uint32_t si = a.list[base + i];
                pw[q] = a.pos[(int64_t)d * a.Mtot + si];
                pt[q] = a.wtab[((int64_t)si * k.D + d) * kWMax + (e % kWMax)];
            }
        }
#pragma unroll
        for (int q = 0; q < kVE; q++) {
            const int e = threadIdx.x + q * kThreads;
            const int i = e / CG, c = e % CG;
            pv[q] = make_float2(0.f, 0.f);
            pd[q] = 1.f;
            if (e < kChunk * CG && i < cnt && b0 + c < a.nb) {
                const uint32_t si = a.list[base + i];
                const uint32_t j = a.perm[si];
                const int64_t idx = (a.layout == LAYOUT_SORTED) ? (int64_t)si : (int64_t)j;
                pv[q] = samples[(int64_t)(b0 + c) * a.Mtot + idx];
                if (a.dcw) pd[q] = a.dcw[j];
            }
        }
        if (threadIdx.x < kChunk) {
            const int i = threadIdx.x;
            for (int d = 0; d < 3; d++)
                ps[d] = (i < cnt && d < k.D) ? a.pos[(int64_t)d * a.Mtot + a.list[base + i]] : 0.f;
        }
    };

    auto stage_chunk = [&](GridStage<CG> &S, int cnt) {
#pragma unroll
        for (int q = 0; q < kWE; q++) {
            const int e = threadIdx.x + q * kThreads;
            if (e >= kChunk * 3 * kWMax) break;
            const int i = e / (3 * kWMax), d = (e / kWMax) % 3, t = e % kWMax;
            float w = 0.f;
            if (i < cnt) {
                if (d < k.D) {
                    const int lo = (int)ceilf(pw[q] - k.radius);
                    w = pt[q];   // zero beyond the footprint
                    if (a.sign_fold) w *= sign_of((lo + t - k.hw) & 1);   // parity of (p - hw) mod mos (mos even)
                } else {
                    w = (t == 0) ? 1.f : 0.f;
                }
            }
            S.w[i][d][t] = w;
        }
#pragma unroll
        for (int q = 0; q < kVE; q++) {
            const int e = threadIdx.x + q * kThreads;
            if (e >= kChunk * CG) break;
            const int i = e / CG, c = e % CG;
            float2 v = pv[q];
            if (a.dcw) {
                v.x = pd[q] * v.x;
                v.y = pd[q] * v.y;
            }
            S.v[i][c] = v;
        }
        if (threadIdx.x < kChunk) {
            const int i = threadIdx.x;
            uint32_t m = 0;
            if (i < cnt) {
                int lo[3], hi[3];
                for (int d = 0; d < 3; d++) {
                    int a_ = 0, n = 1;
                    if (d < k.D) {
                        const float s = ps[d];
                        const int l = (int)ceilf(s - k.radius);
                        n = min((int)floorf(s + k.radius) - l + 1, kWMax);
                        a_ = wrapmod(l - k.hw - org[d], k.mos[d]);
                    }
                    S.a[i][d] = a_;
                    S.n[i][d] = n;
                    const int T = k.tile[d];
                    if (k.ntiles[d] == 1) {   // footprint may wrap inside the tile
                        lo[d] = 0;
                        hi[d] = T - 1;
                    } else {
                        const int st = (a_ < T) ? a_ : a_ - k.mos[d];
                        lo[d] = max(st, 0);
                        hi[d] = min(st + n - 1, T - 1);
                    }
                }
                for (int w = 0; w < 8; w++)
                    for (int c = 0; c < CPT; c++) {
                        const int q = w + 8 * c;
                        const int x0 = (q % npx) * PX, y0 = ((q / npx) % npy) * PY, z0 = q / (npx * npy);
                        if (x0 <= hi[0] && x0 + PX - 1 >= lo[0] && y0 <= hi[1] && y0 + PY - 1 >= lo[1] &&
                            z0 <= hi[2] && z0 >= lo[2])
                            m |= 1u << w;
                    }
            }
            S.mask[i] = m;
        }
    };

    int cur = 0;
    if (it.begin < it.end) {
        const int cnt0 = min(kChunk, it.end - it.begin);
        prefetch(it.begin, cnt0);
        stage_chunk(stage[0], cnt0);
    }
    __syncthreads();
    for (int base = it.begin; base < it.end; base += kChunk) {
        const int cnt = min(kChunk, it.end - base);
        const int nbase = base + kChunk;
        const int ncnt = nbase < it.end ? min(kChunk, it.end - nbase) : 0;
        if (ncnt > 0) prefetch(nbase, ncnt);
        GridStage<CG> &S = stage[cur];
        for (int half = 0; half < kChunk / 32; half++) {
        uint32_t bits = __ballot_sync(0xffffffffu, half * 32 + lane < cnt &&
                                                       ((S.mask[half * 32 + lane] >> warp) & 1u));
        while (bits) {
            const int i = half * 32 + __ffs(bits) - 1;
            bits &= bits - 1;
            const int a0 = S.a[i][0], a1 = S.a[i][1], a2 = S.a[i][2];
            const int n0 = S.n[i][0], n1 = S.n[i][1], n2 = S.n[i][2];
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                int o0 = lc[c][0] - a0; if (o0 < 0) o0 += k.mos[0];
                int o1 = lc[c][1] - a1; if (o1 < 0) o1 += k.mos[1];
                int o2 = lc[c][2] - a2; if (o2 < 0) o2 += k.mos[2];
                if (o0 < n0 && o1 < n1 && o2 < n2) {
                    const float w = (S.w[i][0][o0] * S.w[i][1][o1]) * S.w[i][2][o2];
#pragma unroll
                    for (int q = 0; q < CG; q++) {
                        const float2 v = S.v[i][q];
                        if (COMP) {
                            float y0 = w * v.x - cmp[c][q][0];
                            float t0 = acc[c][q][0] + y0;
                            cmp[c][q][0] = (t0 - acc[c][q][0]) - y0;
                            acc[c][q][0] = t0;
                            float y1 = w * v.y - cmp[c][q][1];
                            float t1 = acc[c][q][1] + y1;
                            cmp[c][q][1] = (t1 - acc[c][q][1]) - y1;
                            acc[c][q][1] = t1;
                        } else {
                            acc[c][q][0] = fmaf(w, v.x, acc[c][q][0]);
                            acc[c][q][1] = fmaf(w, v.y, acc[c][q][1]);
                        }
                    }
                }
            }
        }
        }
        if (ncnt > 0) stage_chunk(stage[cur ^ 1], ncnt);
        __syncthreads();
        cur ^= 1;
    }

    bool cell_ok[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++)
        cell_ok[c] = lc[c][0] < k.tile[0] && lc[c][1] < k.tile[1] && lc[c][2] < k.tile[2];
    auto cell_index = [&](int c) -> int64_t {   // address of the cell within its batch
        const int gx = org[0] + lc[c][0], gy = org[1] + lc[c][1], gz = org[2] + lc[c][2];
        return (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
    };
    if (it.split < 0) {
#pragma unroll
        for (int c = 0; c < CPT; c++) {
            if (!cell_ok[c]) continue;
            const int64_t g = cell_index(c);
#pragma unroll
            for (int q = 0; q < CG; q++) {
                if (b0 + q >= a.nb) break;
                float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * a.kl.s_bf + g;
                float2 v = make_float2(acc[c][q][0], acc[c][q][1]);
                if (a.accumulate) { float2 old = *o; v.x += old.x; v.y += old.y; }
                *o = v;
            }
        }
        return;
    }
    // Split tile: write this chunk's partial, the last CTA reduces in order.
    const SplitInfo si = a.splits[it.split];
    const int cells = kThreads * CPT;
    auto part = [&](int slot) -> float2 * {
        return a.partials + ((int64_t)slot * a.ncg + grp) * (int64_t)CG * cells;
    };
    {
        float2 *pp = part(si.first_slot + it.chunk);
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
            for (int q = 0; q < CG; q++)
                pp[(int64_t)q * cells + c * kThreads + threadIdx.x] = make_float2(acc[c][q][0], acc[c][q][1]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int *ctr = a.counters + (int64_t)it.split * a.ncg + grp;
        unsigned int old = atomicAdd(ctr, 1u);
        s_last = (old == (unsigned int)(si.nchunks - 1));
        if (s_last) *ctr = 0u;   // ready for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        if (!cell_ok[c]) continue;
        const int64_t g = cell_index(c);
#pragma unroll
        for (int q = 0; q < CG; q++) {
            if (b0 + q >= a.nb) break;
            float sr = 0.f, sim = 0.f, cr = 0.f, ci = 0.f;
            for (int ch = 0; ch < si.nchunks; ch++) {
                const float2 v = __ldcg(&part(si.first_slot + ch)[(int64_t)q * cells + c * kThreads + threadIdx.x]);
                if (COMP) {
                    float y0 = v.x - cr, t0 = sr + y0; cr = (t0 - sr) - y0; sr = t0;
                    float y1 = v.y - ci, t1 = sim + y1; ci = (t1 - sim) - y1; sim = t1;
                } else {
                    sr += v.x;
                    sim += v.y;
                }
            }
            float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * a.kl.s_bf + g;
            float2 v = make_float2(sr, sim);
            if (a.accumulate) { float2 old = *o; v.x += old.x; v.y += old.y; }
            *o = v;
        }
    }
}

// ------------------------------------------------- NC2C, row variant -----
//
// Gridding for coil groups of 8 or 16 without compensation.  The tile is cut
// into regions of ROWS x RW cells (ROWS = 64 / CG rows of RW columns, one
// z-slice); warp w owns regions w, w + 8, ... (RPW of them).  A lane is a
// (coil pair, row) of a region and accumulates that row's RW cells for two
// coils in registers, so every lane of a warp works on every sample that
// touches the region.  One visit (sample, region) costs a 16-byte value load,
// the row's y (and z) weight, RW x-weights read as float4 from a per-sample
// weight row laid over the tile (zero outside the footprint) and 4*RW FMAs.
// Sample order per cell is the list order, as in k_grid_nc2c: the result is
// bit-reproducible.

constexpr int kChunkR = 64;   // samples staged per pass (row variant)

// Per stage: the chunk's pair rows (one bulk copy) and its values (sample
// stride cg + 2 float2: an odd number of 16-byte chunks).
__host__ __device__ __forceinline__ int row_stage_bytes(const KParams &k, int cg) {
    return kChunkR * (pair_row_floats(k) * 4 + (cg + 2) * 8);
}

// mbarrier + bulk-copy (TMA) helpers.  Waits are bounded: after ~1 s a wait
// records the failure in *err and waits once more (also bounded) for the copy
// still in flight, then gives up; the results are then wrong but no thread
// spins forever.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned int *err) {
    for (int round = 0; round < 2; round++) {
        for (uint32_t i = 0; i < (1u << 22); i++) {
            if (mbar_try_wait(bar, parity)) return;
            if (i >= 16) __nanosleep(256);
        }
        if (round == 0 && err) atomicOr(err, 1u);
    }
}

template <int CG, int RW, int RPW, bool D3>
__global__ void __launch_bounds__(kThreads, (RPW * RW <= 8) ? 3 : 2)
k_grid_rows(ConvArgs a, const float2 *__restrict__ samples, float2 *__restrict__ grid) {
    constexpr int CP = CG / 2;      // lanes per row: one per coil pair
    constexpr int ROWS = 32 / CP;   // rows per region
    constexpr int SVS = CG + 2;     // staged values: float2 per sample (padded)
    constexpr int kVE = (kChunkR * CG + kThreads - 1) / kThreads;
    extern __shared__ __align__(128) unsigned char g_rows_smem[];
    __shared__ int s_last;

    const KParams &k = a.k;
    const int grp = blockIdx.y;
    const int b0 = grp * CG;
    const WorkItem it = a.items[blockIdx.x];
    const int f = it.ft / k.ntiles_total;
    const int tile = it.ft - f * k.ntiles_total;
    const int tx = tile % k.ntiles[0];
    const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
    const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
    const int org0 = tx * k.tile[0], org1 = ty * k.tile[1], org2 = tz * k.tile[2];
    const int T0 = k.tile[0], T1 = k.tile[1];
    const int PRF = a.prow_floats;   // floats per pair row
    const int PRW = PRF - 4;         // weight part; the last 4 words are the footprint ranges
    const int stage_bytes = row_stage_bytes(k, CG);
    __shared__ __align__(8) unsigned long long s_bar[2];   // one mbarrier per stage

    auto stage_wt = [&](int s) { return reinterpret_cast<float *>(g_rows_smem + s * stage_bytes); };
    auto stage_v = [&](int s) {
        return reinterpret_cast<float2 *>(g_rows_smem + s * stage_bytes + kChunkR * PRF * 4);
    };

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cp = lane % CP, row = lane / CP;
    const int nrx = T0 / RW, nry = T1 / ROWS;
    int qx0[RPW], qy0[RPW], qz[RPW];
#pragma unroll
    for (int c = 0; c < RPW; c++) {
        const int q = warp + 8 * c;
        qx0[c] = (q % nrx) * RW;
        qy0[c] = ((q / nrx) % nry) * ROWS;
        qz[c] = q / (nrx * nry);
    }

    // acc[c][j][h]: (re, im) of coil 2 cp + h at cell j of region c, updated
    // with packed FP32x2 multiply-adds (each component rounds as fmaf).
    float2 acc[RPW][RW][2];
#pragma unroll
    for (int c = 0; c < RPW; c++)
#pragma unroll
        for (int j = 0; j < RW; j++) acc[c][j][0] = acc[c][j][1] = make_float2(0.f, 0.f);

    // A tile no sample touches: its cells are zero (nothing to add when
    // accumulating) -- one pass of coalesced stores, no staging.
    if (it.begin == it.end && it.split < 0) {
        if (a.accumulate) return;
        const int cells = T0 * T1 * k.tile[2];
        const int64_t ostep = (int64_t)a.F * a.kl.s_bf;
        float2 *gbase = grid + ((int64_t)b0 * a.F + f) * a.kl.s_bf;
        for (int e = threadIdx.x; e < cells; e += kThreads) {
            const int x = e % T0, yz = e / T0, y = yz % T1, z = yz / T1;
            float2 *o = gbase + (int64_t)(org2 + z) * a.kl.s_z + (int64_t)(org1 + y) * a.kl.s_y + org0 + x;
            for (int c = 0; c < CG && b0 + c < a.nb; c++) {
                *o = make_float2(0.f, 0.f);
                o += ostep;
            }
        }
        return;
    }

    const uint32_t bar[2] = {smem_u32(&s_bar[0]), smem_u32(&s_bar[1])};
    if (threadIdx.x == 0) {
        mbar_init(bar[0], 1);
        mbar_init(bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase = 0;   // bit s: parity of stage s's next barrier completion

    // The pair rows of a chunk are contiguous (list order): thread 0 starts
    // one bulk copy (TMA) of them into stage s.  Stage s was last read before
    // the preceding __syncthreads; the proxy fence orders those reads before
    // the asynchronous write.
    auto issue_rows = [&](int s, int base, int cnt) {
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            const uint32_t bytes = (uint32_t)cnt * (uint32_t)PRF * 4u;
            mbar_expect_tx(bar[s], bytes);
            bulk_copy_g2s(smem_u32(stage_wt(s)), a.prows + (int64_t)base * PRF, bytes, bar[s]);
        }
    };

    float2 pv[kVE];
    float pd[kVE];
    // values: lanes run along samples (one coil per load instruction)
    auto prefetch = [&](int base, int cnt) {
#pragma unroll
        for (int q = 0; q < kVE; q++) {
            const int e = threadIdx.x + q * kThreads;
            const int i = e % kChunkR, c = e / kChunkR;
            pv[q] = make_float2(0.f, 0.f);
            pd[q] = 1.f;
            if (e < kChunkR * CG && i < cnt && b0 + c < a.nb) {
                const uint32_t si = a.list[base + i];
                const bool need_j = a.layout == LAYOUT_ORIGINAL || a.dcw;
                const uint32_t j = need_j ? a.perm[si] : si;
                const int64_t idx = (a.layout == LAYOUT_SORTED) ? (int64_t)si : (int64_t)j;
                pv[q] = samples[(int64_t)(b0 + c) * a.Mtot + idx];
                if (a.dcw) pd[q] = a.dcw[j];
            }
        }
    };
    // Values of the prefetched chunk into stage s, density weights folded in.
    auto stage_values = [&](int s) {
        float2 *sv = stage_v(s);
#pragma unroll
        for (int q = 0; q < kVE; q++) {
            const int e = threadIdx.x + q * kThreads;
            if (e >= kChunkR * CG) break;
            float2 v = pv[q];
            if (a.dcw) {
                v.x = pd[q] * v.x;
                v.y = pd[q] * v.y;
            }
            sv[(e % kChunkR) * SVS + e / kChunkR] = v;
        }
    };

    int cur = 0;
    if (it.begin < it.end) {
        const int cnt0 = min(kChunkR, it.end - it.begin);
        issue_rows(0, it.begin, cnt0);
        prefetch(it.begin, cnt0);
        stage_values(0);
    }
    __syncthreads();
    for (int base = it.begin; base < it.end; base += kChunkR) {
        const int cnt = min(kChunkR, it.end - base);
        const int nbase = base + kChunkR;
        const int ncnt = nbase < it.end ? min(kChunkR, it.end - nbase) : 0;
        if (ncnt > 0) {
            issue_rows(cur ^ 1, nbase, ncnt);
            prefetch(nbase, ncnt);
        }
        mbar_wait_bounded(bar[cur], (phase >> cur) & 1u, a.err);
        phase ^= 1u << cur;
        const float *wt = stage_wt(cur);
        const float4 *sv4 = reinterpret_cast<const float4 *>(stage_v(cur));
#pragma unroll
        for (int c = 0; c < RPW; c++) {
            const int ry = qy0[c] + row;
#pragma unroll
            for (int half = 0; half < kChunkR / 32; half++) {
                const int il = half * 32 + lane;
                bool hit = false;
                if (il < cnt) {
                    const uint4 r = *reinterpret_cast<const uint4 *>(wt + il * PRF + PRW);
                    hit = (int)(r.x & 0xffffu) <= qx0[c] + RW - 1 && (int)(r.x >> 16) >= qx0[c] &&
                          (int)(r.y & 0xffffu) <= qy0[c] + ROWS - 1 && (int)(r.y >> 16) >= qy0[c];
                    if (D3) hit = hit && (int)(r.z & 0xffffu) <= qz[c] && (int)(r.z >> 16) >= qz[c];
                }
                uint32_t bits = __ballot_sync(0xffffffffu, hit);
                while (bits) {
                    const int i = half * 32 + __ffs(bits) - 1;
                    bits &= bits - 1;
                    const float4 v = sv4[i * (SVS / 2) + cp];
                    const float2 v0 = make_float2(v.x, v.y), v1 = make_float2(v.z, v.w);
                    const float *wr = wt + i * PRF;
                    float wyz = wr[T0 + ry];
                    if (D3) wyz *= wr[T0 + T1 + qz[c]];
                    const float2 wyz2 = make_float2(wyz, wyz);
#pragma unroll
                    for (int jj = 0; jj < RW / 4; jj++) {
                        const float4 w4 = *reinterpret_cast<const float4 *>(wr + qx0[c] + 4 * jj);
                        const float2 w01 = __fmul2_rn(make_float2(w4.x, w4.y), wyz2);
                        const float2 w23 = __fmul2_rn(make_float2(w4.z, w4.w), wyz2);
                        const float wj[4] = {w01.x, w01.y, w23.x, w23.y};
#pragma unroll
                        for (int m = 0; m < 4; m++) {
                            const float2 wm = make_float2(wj[m], wj[m]);
                            float2 *ac = acc[c][4 * jj + m];
                            ac[0] = __ffma2_rn(wm, v0, ac[0]);
                            ac[1] = __ffma2_rn(wm, v1, ac[1]);
                        }
                    }
                }
            }
        }
        if (ncnt > 0) stage_values(cur ^ 1);
        __syncthreads();
        cur ^= 1;
    }

    // The centring checkerboard (-1)^(gx+gy+gz) is a property of the output
    // cell, so it is applied here rather than to every weight.
    auto store = [&](int c, int j, float4 v) {
        const int gx = org0 + qx0[c] + j, gy = org1 + qy0[c] + row, gz = org2 + qz[c];
        const int64_t g = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
        const float sgn = (a.sign_fold && ((gx + gy + gz) & 1)) ? -1.f : 1.f;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int q = 2 * cp + h;
            if (b0 + q >= a.nb) break;
            float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * a.kl.s_bf + g;
            float2 w = h ? make_float2(sgn * v.z, sgn * v.w) : make_float2(sgn * v.x, sgn * v.y);
            if (a.accumulate) { const float2 old = *o; w.x += old.x; w.y += old.y; }
            *o = w;
        }
    };
    // Writes the accumulators to the grid.  Through shared memory when the
    // tile fits the stage buffers: lanes put their cells into a [coil][z][y][x]
    // tile (rows padded by one cell, coil planes to 2 mod 8 cells: conflict-
    // free), then threads store whole rows of one coil plane (coalesced).
    // Every thread of the CTA calls it (it has a barrier).
    auto epilogue = [&]() {
        const int T2 = k.tile[2];
        const int RS = T0 + 1, ZS = T1 * RS;
        int PS = T2 * ZS;
        PS += (10 - PS % 8) % 8;   // PS = 2 (mod 8)
        if ((int64_t)CG * PS * 8 > 2 * (int64_t)stage_bytes) {
#pragma unroll
            for (int c = 0; c < RPW; c++)
#pragma unroll
                for (int j = 0; j < RW; j++)
                    store(c, j, make_float4(acc[c][j][0].x, acc[c][j][0].y, acc[c][j][1].x, acc[c][j][1].y));
            return;
        }
        float2 *tl = reinterpret_cast<float2 *>(g_rows_smem);
#pragma unroll
        for (int c = 0; c < RPW; c++)
#pragma unroll
            for (int j = 0; j < RW; j++) {
                const int o = qz[c] * ZS + (qy0[c] + row) * RS + qx0[c] + j;
                tl[(2 * cp) * PS + o] = acc[c][j][0];
                tl[(2 * cp + 1) * PS + o] = acc[c][j][1];
            }
        __syncthreads();
        const int x = threadIdx.x % T0, r0 = threadIdx.x / T0, rpp = kThreads / T0;
        if (r0 >= rpp) return;
        const int rows_c = T2 * T1;
        const int gx = org0 + x;
        for (int r = r0; r < rows_c; r += rpp) {
            const int z = r / T1, y = r - z * T1;
            const int gy = org1 + y, gz = org2 + z;
            const float sgn = (a.sign_fold && ((gx + gy + gz) & 1)) ? -1.f : 1.f;
            const int64_t cell = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
            const float2 *src = tl + z * ZS + y * RS + x;
            float2 *o = grid + ((int64_t)b0 * a.F + f) * a.kl.s_bf + cell;
            const int64_t ostep = (int64_t)a.F * a.kl.s_bf;
            for (int c = 0; c < CG && b0 + c < a.nb; c++) {
                float2 v = src[c * PS];
                v.x *= sgn;
                v.y *= sgn;
                if (a.accumulate) { const float2 old = *o; v.x += old.x; v.y += old.y; }
                *o = v;
                o += ostep;
            }
        }
    };
    if (it.split < 0) {
        epilogue();
        return;
    }
    // Split tile: write this chunk's partial tile, the last CTA sums the
    // partials in chunk order.
    const SplitInfo si = a.splits[it.split];
    auto part = [&](int slot) -> float4 * {
        return reinterpret_cast<float4 *>(a.partials + ((int64_t)slot * a.ncg + grp) * a.part_elems);
    };
    {
        float4 *pp = part(si.first_slot + it.chunk);
#pragma unroll
        for (int c = 0; c < RPW; c++)
#pragma unroll
            for (int j = 0; j < RW; j++)
                pp[(c * RW + j) * kThreads + threadIdx.x] =
                    make_float4(acc[c][j][0].x, acc[c][j][0].y, acc[c][j][1].x, acc[c][j][1].y);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int *ctr = a.counters + (int64_t)it.split * a.ncg + grp;
        const unsigned int old = atomicAdd(ctr, 1u);
        s_last = (old == (unsigned int)(si.nchunks - 1));
        if (s_last) *ctr = 0u;   // ready for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int c = 0; c < RPW; c++)
#pragma unroll
        for (int j = 0; j < RW; j++) {
            float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int ch = 0; ch < si.nchunks; ch++) {
                const float4 v = __ldcg(&part(si.first_slot + ch)[(c * RW + j) * kThreads + threadIdx.x]);
                s.x += v.x;
                s.y += v.y;
                s.z += v.z;
                s.w += v.w;
            }
            acc[c][j][0] = make_float2(s.x, s.y);
            acc[c][j][1] = make_float2(s.z, s.w);
        }
    epilogue();
}

// ------------------------------------- NC2C, row variant, warp-specialized --
//
// The row variant for SORTED_IL samples (the E^H E workspace, where every
// sample's coils are one contiguous row).  Nothing is staged through
// registers: a producer warp (warp 8) streams each chunk's pair rows and
// sample rows into a ring of kWsStages shared-memory stages with bulk copies
// (cp.async.bulk), announcing the bytes on the stage's "full" mbarrier; the
// eight consumer warps run the same region visits as k_grid_rows and release
// a stage on its "empty" mbarrier (one arrival per warp) when done with it.
// Warps never wait for each other inside the chunk loop, and the copies of
// the next kWsStages - 1 chunks are in flight while a chunk is summed.  All
// waits are bounded (err bit 0).  Same per-cell summation order as
// k_grid_rows, so the result is bit-identical.

constexpr int kWsStages = 4;
constexpr int kWsThreads = kThreads + 32;   // 8 consumer warps + 1 producer warp
constexpr int kWsMinBlocks = 2;             // resident CTAs per SM (96 registers a thread)

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

__host__ __device__ __forceinline__ int ws_stage_bytes(const KParams &k, int cg) {
    return kChunkR * (pair_row_floats(k) * 4 + cg * 8);
}

template <int CG, int RW, int RPW, bool D3>
__global__ void __launch_bounds__(kWsThreads, kWsMinBlocks)
k_grid_rows_ws(ConvArgs a, const float2 *__restrict__ samples, float2 *__restrict__ grid) {
    constexpr int CP = CG / 2;      // lanes per row: one per coil pair
    constexpr int ROWS = 32 / CP;   // rows per region
    extern __shared__ __align__(128) unsigned char g_ws_smem[];
    __shared__ int s_last;
    __shared__ __align__(8) unsigned long long s_full[kWsStages], s_empty[kWsStages];

    const KParams &k = a.k;
    const int grp = blockIdx.y;
    const int b0 = grp * CG;
    const WorkItem it = a.items[blockIdx.x];
    const int f = it.ft / k.ntiles_total;
    const int tile = it.ft - f * k.ntiles_total;
    const int tx = tile % k.ntiles[0];
    const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
    const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
    const int org0 = tx * k.tile[0], org1 = ty * k.tile[1], org2 = tz * k.tile[2];
    const int T0 = k.tile[0], T1 = k.tile[1];
    const int PRF = a.prow_floats;   // floats per pair row
    const int PRW = PRF - 4;         // weight part; the last 4 words are the footprint ranges
    const int stage_bytes = ws_stage_bytes(k, CG);
    auto stage_wt = [&](int s) { return reinterpret_cast<float *>(g_ws_smem + s * stage_bytes); };
    auto stage_v = [&](int s) {
        return reinterpret_cast<float2 *>(g_ws_smem + s * stage_bytes + kChunkR * PRF * 4);
    };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool consumer = warp < 8;

    // A tile no sample touches: zero stores, no staging.
    if (it.begin == it.end && it.split < 0) {
        if (a.accumulate) return;
        const int cells = T0 * T1 * k.tile[2];
        const int64_t ostep = (int64_t)a.F * a.kl.s_bf;
        float2 *gbase = grid + ((int64_t)b0 * a.F + f) * a.kl.s_bf;
        for (int e = threadIdx.x; e < cells; e += blockDim.x) {
            const int x = e % T0, yz = e / T0, y = yz % T1, z = yz / T1;
            float2 *o = gbase + (int64_t)(org2 + z) * a.kl.s_z + (int64_t)(org1 + y) * a.kl.s_y + org0 + x;
            for (int c = 0; c < CG && b0 + c < a.nb; c++) {
                *o = make_float2(0.f, 0.f);
                o += ostep;
            }
        }
        return;
    }

    if (threadIdx.x == 0) {
        for (int st = 0; st < kWsStages; st++) {
            mbar_init(smem_u32(&s_full[st]), 1);
            mbar_init(smem_u32(&s_empty[st]), 8);
        }
        mbar_fence_init();
    }
    __syncthreads();
    const int nchunks = (it.end - it.begin + kChunkR - 1) / kChunkR;

    const int cp = lane % CP, row = lane / CP;
    const int nrx = T0 / RW, nry = T1 / ROWS;
    int qx0[RPW], qy0[RPW], qz[RPW];
#pragma unroll
    for (int c = 0; c < RPW; c++) {
        const int q = (consumer ? warp : 0) + 8 * c;
        qx0[c] = (q % nrx) * RW;
        qy0[c] = ((q / nrx) % nry) * ROWS;
        qz[c] = q / (nrx * nry);
    }
    float2 acc[RPW][RW][2];
#pragma unroll
    for (int c = 0; c < RPW; c++)
#pragma unroll
        for (int j = 0; j < RW; j++) acc[c][j][0] = acc[c][j][1] = make_float2(0.f, 0.f);

    if (!consumer) {
        // Producer: for chunk ch, stage ch % kWsStages once the consumers
        // released its previous use; lane 0 announces all bytes (arrival +
        // transaction count) and copies the pair rows, then every lane copies
        // up to two sample rows (this coil group's columns).
        const uint32_t vbytes = (uint32_t)min(CG, a.il_stride - b0) * 8u;
        for (int ch = 0; ch < nchunks; ch++) {
            const int st = ch % kWsStages;
            const int use = ch / kWsStages;
            const int base = it.begin + ch * kChunkR;
            const int cnt = min(kChunkR, it.end - base);
            const uint32_t si0 = lane < cnt ? a.list[base + lane] : 0u;
            const uint32_t si1 = lane + 32 < cnt ? a.list[base + lane + 32] : 0u;
            if (use > 0) mbar_wait_bounded(smem_u32(&s_empty[st]), (uint32_t)(use - 1) & 1u, a.err);
            fence_proxy_async_smem();
            const uint32_t full = smem_u32(&s_full[st]);
            if (lane == 0) {
                const uint32_t rbytes = (uint32_t)cnt * (uint32_t)PRF * 4u;
                mbar_expect_tx(full, rbytes + (uint32_t)cnt * vbytes);
                bulk_copy_g2s(smem_u32(stage_wt(st)), a.prows + (int64_t)base * PRF, rbytes, full);
            }
            __syncwarp();
            float2 *sv = stage_v(st);
            if (lane < cnt)
                bulk_copy_g2s(smem_u32(sv + lane * CG), samples + (int64_t)si0 * a.il_stride + b0, vbytes, full);
            if (lane + 32 < cnt)
                bulk_copy_g2s(smem_u32(sv + (lane + 32) * CG), samples + (int64_t)si1 * a.il_stride + b0, vbytes,
                              full);
        }
    } else {
        for (int ch = 0; ch < nchunks; ch++) {
            const int st = ch % kWsStages;
            const int base = it.begin + ch * kChunkR;
            const int cnt = min(kChunkR, it.end - base);
            mbar_wait_bounded(smem_u32(&s_full[st]), (uint32_t)(ch / kWsStages) & 1u, a.err);
            const float *wt = stage_wt(st);
            const float4 *sv4 = reinterpret_cast<const float4 *>(stage_v(st));
#pragma unroll
            for (int c = 0; c < RPW; c++) {
                const int ry = qy0[c] + row;
#pragma unroll
                for (int half = 0; half < kChunkR / 32; half++) {
                    const int il = half * 32 + lane;
                    bool hit = false;
                    if (il < cnt) {
                        const uint4 r = *reinterpret_cast<const uint4 *>(wt + il * PRF + PRW);
                        hit = (int)(r.x & 0xffffu) <= qx0[c] + RW - 1 && (int)(r.x >> 16) >= qx0[c] &&
                              (int)(r.y & 0xffffu) <= qy0[c] + ROWS - 1 && (int)(r.y >> 16) >= qy0[c];
                        if (D3) hit = hit && (int)(r.z & 0xffffu) <= qz[c] && (int)(r.z >> 16) >= qz[c];
                    }
                    uint32_t bits = __ballot_sync(0xffffffffu, hit);
                    while (bits) {
                        const int i = half * 32 + __ffs(bits) - 1;
                        bits &= bits - 1;
                        const float4 v = sv4[i * (CG / 2) + cp];
                        const float2 v0 = make_float2(v.x, v.y), v1 = make_float2(v.z, v.w);
                        const float *wr = wt + i * PRF;
                        float wyz = wr[T0 + ry];
                        if (D3) wyz *= wr[T0 + T1 + qz[c]];
                        const float2 wyz2 = make_float2(wyz, wyz);
#pragma unroll
                        for (int jj = 0; jj < RW / 4; jj++) {
                            const float4 w4 = *reinterpret_cast<const float4 *>(wr + qx0[c] + 4 * jj);
                            const float2 w01 = __fmul2_rn(make_float2(w4.x, w4.y), wyz2);
                            const float2 w23 = __fmul2_rn(make_float2(w4.z, w4.w), wyz2);
                            const float wj[4] = {w01.x, w01.y, w23.x, w23.y};
#pragma unroll
                            for (int m = 0; m < 4; m++) {
                                const float2 wm = make_float2(wj[m], wj[m]);
                                float2 *ac = acc[c][4 * jj + m];
                                ac[0] = __ffma2_rn(wm, v0, ac[0]);
                                ac[1] = __ffma2_rn(wm, v1, ac[1]);
                            }
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&s_empty[st]));
        }
    }
    __syncthreads();   // every stage consumed; every copy landed

    auto store = [&](int c, int j, float4 v) {
        const int gx = org0 + qx0[c] + j, gy = org1 + qy0[c] + row, gz = org2 + qz[c];
        const int64_t g = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
        const float sgn = (a.sign_fold && ((gx + gy + gz) & 1)) ? -1.f : 1.f;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int q = 2 * cp + h;
            if (b0 + q >= a.nb) break;
            float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * a.kl.s_bf + g;
            float2 w = h ? make_float2(sgn * v.z, sgn * v.w) : make_float2(sgn * v.x, sgn * v.y);
            if (a.accumulate) { const float2 old = *o; w.x += old.x; w.y += old.y; }
            *o = w;
        }
    };
    // Tile out through shared memory (as k_grid_rows), the stage ring as the
    // staging area.  Every thread calls it (it has a barrier).
    auto epilogue = [&]() {
        const int T2 = k.tile[2];
        const int RS = T0 + 1, ZS = T1 * RS;
        int PS = T2 * ZS;
        PS += (10 - PS % 8) % 8;   // PS = 2 (mod 8)
        if ((int64_t)CG * PS * 8 > (int64_t)kWsStages * stage_bytes) {
            if (consumer) {
#pragma unroll
                for (int c = 0; c < RPW; c++)
#pragma unroll
                    for (int j = 0; j < RW; j++)
                        store(c, j, make_float4(acc[c][j][0].x, acc[c][j][0].y, acc[c][j][1].x, acc[c][j][1].y));
            }
            return;
        }
        float2 *tl = reinterpret_cast<float2 *>(g_ws_smem);
        if (consumer) {
#pragma unroll
            for (int c = 0; c < RPW; c++)
#pragma unroll
                for (int j = 0; j < RW; j++) {
                    const int o = qz[c] * ZS + (qy0[c] + row) * RS + qx0[c] + j;
                    tl[(2 * cp) * PS + o] = acc[c][j][0];
                    tl[(2 * cp + 1) * PS + o] = acc[c][j][1];
                }
        }
        __syncthreads();
        const int x = threadIdx.x % T0, r0 = threadIdx.x / T0, rpp = kThreads / T0;
        if (r0 >= rpp) return;
        const int rows_c = T2 * T1;
        const int gx = org0 + x;
        for (int r = r0; r < rows_c; r += rpp) {
            const int z = r / T1, y = r - z * T1;
            const int gy = org1 + y, gz = org2 + z;
            const float sgn = (a.sign_fold && ((gx + gy + gz) & 1)) ? -1.f : 1.f;
            const int64_t cell = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
            const float2 *src = tl + z * ZS + y * RS + x;
            float2 *o = grid + ((int64_t)b0 * a.F + f) * a.kl.s_bf + cell;
            const int64_t ostep = (int64_t)a.F * a.kl.s_bf;
            for (int c = 0; c < CG && b0 + c < a.nb; c++) {
                float2 v = src[c * PS];
                v.x *= sgn;
                v.y *= sgn;
                if (a.accumulate) { const float2 old = *o; v.x += old.x; v.y += old.y; }
                *o = v;
                o += ostep;
            }
        }
    };
    if (it.split < 0) {
        epilogue();
        return;
    }
    // Split tile: write this chunk's partial tile, the last CTA sums the
    // partials in chunk order.
    const SplitInfo si = a.splits[it.split];
    auto part = [&](int slot) -> float4 * {
        return reinterpret_cast<float4 *>(a.partials + ((int64_t)slot * a.ncg + grp) * a.part_elems);
    };
    if (consumer) {
        float4 *pp = part(si.first_slot + it.chunk);
#pragma unroll
        for (int c = 0; c < RPW; c++)
#pragma unroll
            for (int j = 0; j < RW; j++)
                pp[(c * RW + j) * kThreads + threadIdx.x] =
                    make_float4(acc[c][j][0].x, acc[c][j][0].y, acc[c][j][1].x, acc[c][j][1].y);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int *ctr = a.counters + (int64_t)it.split * a.ncg + grp;
        const unsigned int old = atomicAdd(ctr, 1u);
        s_last = (old == (unsigned int)(si.nchunks - 1));
        if (s_last) *ctr = 0u;   // ready for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (consumer) {
#pragma unroll
        for (int c = 0; c < RPW; c++)
#pragma unroll
            for (int j = 0; j < RW; j++) {
                float4 sm = make_float4(0.f, 0.f, 0.f, 0.f);
                for (int ch = 0; ch < si.nchunks; ch++) {
                    const float4 v = __ldcg(&part(si.first_slot + ch)[(c * RW + j) * kThreads + threadIdx.x]);
                    sm.x += v.x;
                    sm.y += v.y;
                    sm.z += v.z;
                    sm.w += v.w;
                }
                acc[c][j][0] = make_float2(sm.x, sm.y);
                acc[c][j][1] = make_float2(sm.z, sm.w);
            }
    }
    epilogue();
}

// ---------------------- NC2C, row variant, warp-specialized, persistent --
//
// k_grid_rows_ws as one persistent launch over every work unit (gridding
// item x coil group) of all frames: kWsMinBlocks CTAs per SM take units from
// a global counter (units in list order: split chunks of heavy tiles first),
// and the producer warp streams chunk after chunk across unit boundaries, so
// the copy pipeline does not drain between tiles and no CTA pays a launch
// ramp per tile.  Every stage carries a descriptor of its chunk (unit, sample
// count, first/last flags); the consumer warps zero their accumulators on a
// unit's first chunk and write the tile out after its last one, through a
// tile buffer of their own (the producer keeps filling stages meanwhile),
// synchronising only among themselves (an mbarrier of the 256 consumer
// threads).  No CTA waits for another; the last CTA to finish resets the
// counter for the next launch.  Every wait is bounded: a wait that runs out
// sets err bit 0 and the CTA's bail flag, after which every wait of the CTA
// returns at once, both loops end, and the producer waits (bounded) for its
// copies still in flight before the CTA exits.  Per-cell summation order as
// k_grid_rows: the result is bit-identical.

struct WspDesc {
    int ft, split, chunk, grp;
    int cnt, flags, pad0, pad1;
};
constexpr int kWspFirst = 1, kWspLast = 2, kWspDone = 4, kWspEmpty = 8;

// Bounded wait that reports whether the phase completed.  It gives up after
// ~2 s (err bit 0 and *bail set) or as soon as *bail is set (bail may be null).
__device__ __forceinline__ bool mbar_wait_ok(uint32_t bar, uint32_t parity, unsigned int *err, int *bail) {
    for (int round = 0; round < 2; round++) {
        for (uint32_t i = 0; i < (1u << 22); i++) {
            if (mbar_try_wait(bar, parity)) return true;
            if (bail && *reinterpret_cast<volatile int *>(bail)) return false;
            if (i >= 16) __nanosleep(256);
        }
    }
    if (err) atomicOr(err, 1u);
    if (bail) *reinterpret_cast<volatile int *>(bail) = 1;
    return false;
}

// Epilogue tile of the persistent kernel: [coil][z][y][x], rows padded by
// one cell, coil planes at 2 (mod 8) cells (conflict-free transposition).
__host__ __device__ __forceinline__ int wsp_plane_cells(const KParams &k) {
    const int ps = k.tile[2] * k.tile[1] * (k.tile[0] + 1);
    return ps + (10 - ps % 8) % 8;
}
__host__ __device__ __forceinline__ int wsp_smem_bytes(const KParams &k, int cg) {
    return kWsStages * ws_stage_bytes(k, cg) + cg * wsp_plane_cells(k) * 8;
}

template <int CG, int RW, int RPW, bool D3>
__global__ void __launch_bounds__(kWsThreads, kWsMinBlocks)
k_grid_rows_wsp(ConvArgs a, const float2 *__restrict__ samples, float2 *__restrict__ grid) {
    constexpr int CP = CG / 2;      // lanes per row: one per coil pair
    constexpr int ROWS = 32 / CP;   // rows per region
    extern __shared__ __align__(128) unsigned char g_wsp_smem[];
    __shared__ int s_last, s_bail;
    __shared__ __align__(8) unsigned long long s_full[kWsStages], s_empty[kWsStages], s_cons[2];
    __shared__ WspDesc s_desc[kWsStages];

    const KParams &k = a.k;
    const int T0 = k.tile[0], T1 = k.tile[1], T2 = k.tile[2];
    const int PRF = a.prow_floats;   // floats per pair row
    const int PRW = PRF - 4;         // weight part; the last 4 words are the footprint ranges
    const int stage_bytes = ws_stage_bytes(k, CG);
    auto stage_wt = [&](int s) { return reinterpret_cast<float *>(g_wsp_smem + s * stage_bytes); };
    auto stage_v = [&](int s) {
        return reinterpret_cast<float2 *>(g_wsp_smem + s * stage_bytes + kChunkR * PRF * 4);
    };
    float2 *tl = reinterpret_cast<float2 *>(g_wsp_smem + kWsStages * stage_bytes);
    const int PS = wsp_plane_cells(k);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool consumer = warp < 8;

    if (threadIdx.x == 0) {
        for (int st = 0; st < kWsStages; st++) {
            mbar_init(smem_u32(&s_full[st]), 1);
            mbar_init(smem_u32(&s_empty[st]), 8);
        }
        mbar_init(smem_u32(&s_cons[0]), kThreads);
        mbar_init(smem_u32(&s_cons[1]), kThreads);
        mbar_fence_init();
        s_bail = 0;
    }
    __syncthreads();

    if (!consumer) {
        // Producer: takes units from the counter (the next one is fetched
        // while the current one's chunks are issued); for chunk g of the
        // CTA's sequence, stage g % kWsStages once the consumers released its
        // previous use: lane 0 writes the descriptor, announces the bytes
        // (arrival + transaction count) and copies the pair rows, then every
        // lane copies up to two sample rows (this coil group's columns).  A
        // last descriptor flagged kWspDone ends the consumers' loop.
        const int ncg = a.ncg;
        uint32_t g = 0;
        int w = 0;
        if (lane == 0) w = (int)atomicAdd(&a.queue[0], 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        bool bail = false;
        while (!bail) {
            const bool done = w >= a.n_work;
            int wn = w;
            if (!done) {
                if (lane == 0) wn = (int)atomicAdd(&a.queue[0], 1u);
                wn = __shfl_sync(0xffffffffu, wn, 0);
            }
            WorkItem it{};
            int grp = 0;
            if (!done) {
                it = a.items[w / ncg];
                grp = w - (w / ncg) * ncg;
            }
            const int b0 = grp * CG;
            const int n = done ? 0 : it.end - it.begin;
            const uint32_t vbytes = n > 0 ? (uint32_t)min(CG, a.il_stride - b0) * 8u : 0u;
            const int nch = n > 0 ? (n + kChunkR - 1) / kChunkR : 1;
            for (int ch = 0; ch < nch; ch++, g++) {
                const int st = (int)(g % kWsStages);
                const uint32_t use = g / kWsStages;
                const int base = it.begin + ch * kChunkR;
                const int cnt = n > 0 ? min(kChunkR, it.end - base) : 0;
                const uint32_t si0 = lane < cnt ? a.list[base + lane] : 0u;
                const uint32_t si1 = lane + 32 < cnt ? a.list[base + lane + 32] : 0u;
                if (use > 0 && !mbar_wait_ok(smem_u32(&s_empty[st]), (use - 1) & 1u, a.err, &s_bail)) bail = true;
                if (*reinterpret_cast<volatile int *>(&s_bail)) bail = true;
                if (bail) break;
                const uint32_t full = smem_u32(&s_full[st]);
                if (lane == 0) {
                    WspDesc d;
                    d.ft = it.ft;
                    d.split = it.split;
                    d.chunk = it.chunk;
                    d.grp = grp;
                    d.cnt = cnt;
                    d.flags = (ch == 0 ? kWspFirst : 0) | (ch == nch - 1 ? kWspLast : 0) | (done ? kWspDone : 0) |
                              (n == 0 ? kWspEmpty : 0);
                    d.pad0 = d.pad1 = 0;
                    s_desc[st] = d;
                }
                fence_proxy_async_smem();
                if (lane == 0) {
                    const uint32_t rbytes = (uint32_t)cnt * (uint32_t)PRF * 4u;
                    if (cnt > 0) {
                        mbar_expect_tx(full, rbytes + (uint32_t)cnt * vbytes);
                        bulk_copy_g2s(smem_u32(stage_wt(st)), a.prows + (int64_t)base * PRF, rbytes, full);
                    } else {
                        mbar_arrive(full);
                    }
                }
                __syncwarp();
                float2 *sv = stage_v(st);
                if (lane < cnt)
                    bulk_copy_g2s(smem_u32(sv + lane * CG), samples + (int64_t)si0 * a.il_stride + b0, vbytes, full);
                if (lane + 32 < cnt)
                    bulk_copy_g2s(smem_u32(sv + (lane + 32) * CG), samples + (int64_t)si1 * a.il_stride + b0,
                                  vbytes, full);
            }
            if (done) break;
            w = wn;
        }
        if (bail) {
            // the consumers stopped early: wait for the copies still in flight
            for (uint32_t gi = g > kWsStages ? g - kWsStages : 0; gi < g; gi++)
                mbar_wait_ok(smem_u32(&s_full[gi % kWsStages]), (gi / kWsStages) & 1u, nullptr, nullptr);
        }
    } else {
        const int cp = lane % CP, row = lane / CP;
        const int nrx = T0 / RW, nry = T1 / ROWS;
        int qx0[RPW], qy0[RPW], qz[RPW];
#pragma unroll
        for (int c = 0; c < RPW; c++) {
            const int q = warp + 8 * c;
            qx0[c] = (q % nrx) * RW;
            qy0[c] = ((q / nrx) % nry) * ROWS;
            qz[c] = q / (nrx * nry);
        }
        float2 acc[RPW][RW][2];
#pragma unroll
        for (int c = 0; c < RPW; c++)
#pragma unroll
            for (int j = 0; j < RW; j++) acc[c][j][0] = acc[c][j][1] = make_float2(0.f, 0.f);

        // Barrier of the 256 consumer threads (every thread arrives: its
        // shared-memory writes are released to the others).
        uint32_t ncs = 0;
        auto consumer_bar = [&]() {
            const uint32_t b = smem_u32(&s_cons[ncs & 1u]);
            mbar_arrive(b);
            mbar_wait_ok(b, (ncs >> 1) & 1u, a.err, &s_bail);
            ncs++;
        };
        // Tile out through the tile buffer: lanes put their cells into the
        // [coil][z][y][x] tile, then the 256 consumer threads store whole rows
        // of one coil plane (coalesced).
        auto epilogue = [&](int f, int org0, int org1, int org2, int b0) {
            const int RS = T0 + 1, ZS = T1 * RS;
            consumer_bar();   // the previous tile has left the buffer
#pragma unroll
            for (int c = 0; c < RPW; c++)
#pragma unroll
                for (int j = 0; j < RW; j++) {
                    const int o = qz[c] * ZS + (qy0[c] + row) * RS + qx0[c] + j;
                    tl[(2 * cp) * PS + o] = acc[c][j][0];
                    tl[(2 * cp + 1) * PS + o] = acc[c][j][1];
                }
            consumer_bar();
            const int x = threadIdx.x % T0, r0 = threadIdx.x / T0, rpp = kThreads / T0;
            if (r0 >= rpp) return;
            const int rows_c = T2 * T1;
            const int gx = org0 + x;
            const int64_t ostep = (int64_t)a.F * a.kl.s_bf;
            for (int r = r0; r < rows_c; r += rpp) {
                const int z = r / T1, y = r - z * T1;
                const int gy = org1 + y, gz = org2 + z;
                const float sgn = (a.sign_fold && ((gx + gy + gz) & 1)) ? -1.f : 1.f;
                const int64_t cell = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
                const float2 *src = tl + z * ZS + y * RS + x;
                float2 *o = grid + ((int64_t)b0 * a.F + f) * a.kl.s_bf + cell;
                for (int c = 0; c < CG && b0 + c < a.nb; c++) {
                    float2 v = src[c * PS];
                    v.x *= sgn;
                    v.y *= sgn;
                    if (a.accumulate) { const float2 old = *o; v.x += old.x; v.y += old.y; }
                    *o = v;
                    o += ostep;
                }
            }
        };

        uint32_t g = 0;
        for (;;) {
            const int st = (int)(g % kWsStages);
            if (!mbar_wait_ok(smem_u32(&s_full[st]), (g / kWsStages) & 1u, a.err, &s_bail)) break;
            const WspDesc d = s_desc[st];
            if (d.flags & kWspDone) break;
            if (d.flags & kWspFirst) {
#pragma unroll
                for (int c = 0; c < RPW; c++)
#pragma unroll
                    for (int j = 0; j < RW; j++) acc[c][j][0] = acc[c][j][1] = make_float2(0.f, 0.f);
            }
            const int cnt = d.cnt;
            const float *wt = stage_wt(st);
            const float4 *sv4 = reinterpret_cast<const float4 *>(stage_v(st));
#pragma unroll
            for (int c = 0; c < RPW; c++) {
                const int ry = qy0[c] + row;
#pragma unroll
                for (int half = 0; half < kChunkR / 32; half++) {
                    const int il = half * 32 + lane;
                    bool hit = false;
                    if (il < cnt) {
                        const uint4 r = *reinterpret_cast<const uint4 *>(wt + il * PRF + PRW);
                        hit = (int)(r.x & 0xffffu) <= qx0[c] + RW - 1 && (int)(r.x >> 16) >= qx0[c] &&
                              (int)(r.y & 0xffffu) <= qy0[c] + ROWS - 1 && (int)(r.y >> 16) >= qy0[c];
                        if (D3) hit = hit && (int)(r.z & 0xffffu) <= qz[c] && (int)(r.z >> 16) >= qz[c];
                    }
                    uint32_t bits = __ballot_sync(0xffffffffu, hit);
                    while (bits) {
                        const int i = half * 32 + __ffs(bits) - 1;
                        bits &= bits - 1;
                        const float4 v = sv4[i * (CG / 2) + cp];
                        const float2 v0 = make_float2(v.x, v.y), v1 = make_float2(v.z, v.w);
                        const float *wr = wt + i * PRF;
                        float wyz = wr[T0 + ry];
                        if (D3) wyz *= wr[T0 + T1 + qz[c]];
                        const float2 wyz2 = make_float2(wyz, wyz);
#pragma unroll
                        for (int jj = 0; jj < RW / 4; jj++) {
                            const float4 w4 = *reinterpret_cast<const float4 *>(wr + qx0[c] + 4 * jj);
                            const float2 w01 = __fmul2_rn(make_float2(w4.x, w4.y), wyz2);
                            const float2 w23 = __fmul2_rn(make_float2(w4.z, w4.w), wyz2);
                            const float wj[4] = {w01.x, w01.y, w23.x, w23.y};
#pragma unroll
                            for (int m = 0; m < 4; m++) {
                                const float2 wm = make_float2(wj[m], wj[m]);
                                float2 *ac = acc[c][4 * jj + m];
                                ac[0] = __ffma2_rn(wm, v0, ac[0]);
                                ac[1] = __ffma2_rn(wm, v1, ac[1]);
                            }
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&s_empty[st]));
            g++;
            if (!(d.flags & kWspLast)) continue;

            // The unit's tile is complete in the accumulators.
            const int f = d.ft / k.ntiles_total;
            const int tile = d.ft - f * k.ntiles_total;
            const int tx = tile % k.ntiles[0];
            const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
            const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
            const int org0 = tx * T0, org1 = ty * T1, org2 = tz * T2;
            const int b0 = d.grp * CG;
            if (d.split < 0) {
                if (!((d.flags & kWspEmpty) && a.accumulate)) epilogue(f, org0, org1, org2, b0);
                continue;
            }
            // Split tile: write this chunk's partial tile, the last CTA to
            // finish one sums the partials in chunk order.
            const SplitInfo si = a.splits[d.split];
            auto part = [&](int slot) -> float4 * {
                return reinterpret_cast<float4 *>(a.partials + ((int64_t)slot * a.ncg + d.grp) * a.part_elems);
            };
            {
                float4 *pp = part(si.first_slot + d.chunk);
#pragma unroll
                for (int c = 0; c < RPW; c++)
#pragma unroll
                    for (int j = 0; j < RW; j++)
                        pp[(c * RW + j) * kThreads + threadIdx.x] =
                            make_float4(acc[c][j][0].x, acc[c][j][0].y, acc[c][j][1].x, acc[c][j][1].y);
            }
            __threadfence();
            consumer_bar();
            if (threadIdx.x == 0) {
                unsigned int *ctr = a.counters + (int64_t)d.split * a.ncg + d.grp;
                const unsigned int old = atomicAdd(ctr, 1u);
                s_last = (old == (unsigned int)(si.nchunks - 1));
                if (s_last) *ctr = 0u;   // ready for the next launch
            }
            consumer_bar();
            if (!*reinterpret_cast<volatile int *>(&s_last)) continue;
            __threadfence();
#pragma unroll
            for (int c = 0; c < RPW; c++)
#pragma unroll
                for (int j = 0; j < RW; j++) {
                    float4 sm = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (int ch = 0; ch < si.nchunks; ch++) {
                        const float4 v = __ldcg(&part(si.first_slot + ch)[(c * RW + j) * kThreads + threadIdx.x]);
                        sm.x += v.x;
                        sm.y += v.y;
                        sm.z += v.z;
                        sm.w += v.w;
                    }
                    acc[c][j][0] = make_float2(sm.x, sm.y);
                    acc[c][j][1] = make_float2(sm.z, sm.w);
                }
            epilogue(f, org0, org1, org2, b0);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int old = atomicAdd(&a.queue[1], 1u);
        if (old == gridDim.x - 1) {   // every CTA has taken its last unit
            a.queue[0] = 0u;
            a.queue[1] = 0u;
            __threadfence();
        }
    }
}

// ------------------------------------------ reference fold (3D, opt-in) --
//
// GB_FLAG_REFERENCE_FOLD.  The reference grids onto a padded grid and folds
// the ring back in wrap_image_kernel (ConvolverNC2C_standard.cuh:394-437):
// for each nonempty combination of dimensions it tries the 2^d wrap
// directions and adds the first periodic image whose dimensions all wrap.
// It tests whether dimension i (1-based) belongs to a combination with
// `i & combination` (:411-413), which for i = 3 looks at bits 0|1 instead of
// bit 2.  ref_fold_mult() restates that loop: how many times the periodic
// image at shift sigma (per dimension -1, 0, +1) is added to a cell in state
// st (per dimension 0 inside, 1 within the ring width of the low face, 2 of
// the high face).  It is 1 everywhere in 1D and 2D, and in 3D differs from 1
// only on cells within the ring width of a z face.  The periodic gridding
// counts every image once, so after it k_ref_fold_fix adds (mult - 1) times
// each wrapped tap's contribution (float atomics: few taps -- only samples
// whose footprint crosses the grid's edge have wrapped taps).
__device__ int ref_fold_mult(int D, const int *st, const int *sigma) {
    bool zero = true;
    for (int d = 0; d < D; d++) zero &= sigma[d] == 0;
    if (zero) return 1;
    int count = 0;
    for (int comb = 1; comb < (1 << D); comb++) {
        int nd = 0;
        for (int i = 0; i < D; i++) nd += (comb & (1 << i)) != 0;
        for (int sel = 0; sel < (1 << nd); sel++) {
            int stride[kMaxD] = {0, 0, 0}, wraps = 0, skipped = 0;
            for (int i = 1; i <= D; i++) {
                if (i & comb) {
                    if (i & (sel << skipped)) {
                        if (st[i - 1] == 2) { stride[i - 1] = -1; wraps++; }
                    } else {
                        if (st[i - 1] == 1) { stride[i - 1] = 1; wraps++; }
                    }
                } else {
                    skipped++;
                }
            }
            if (wraps == nd) {
                bool same = true;
                for (int d = 0; d < D; d++) same &= stride[d] == sigma[d];
                count += same ? 1 : 0;
                break;
            }
        }
    }
    return count;
}

// One thread per sorted sample; samples whose footprint stays inside the
// grid return at once.
__global__ void k_ref_fold_fix(ConvArgs a, const float2 *__restrict__ samples, float2 *__restrict__ grid) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const KParams &k = a.k;
    if (j >= a.Mtot) return;
    int lo[3], n[3];
    bool crosses = false;
    for (int d = 0; d < 3; d++) {
        const float s = a.pos[(int64_t)d * a.Mtot + j];
        lo[d] = (int)ceilf(s - k.radius);
        n[d] = min((int)floorf(s + k.radius) - lo[d] + 1, kWMax);
        const int u0 = lo[d] - k.hw, u1 = u0 + n[d] - 1;
        crosses |= u0 < 0 || u1 >= k.mos[d];
    }
    if (!crosses) return;
    const int f = (int)(a.home_key[j] / (uint32_t)k.ntiles_total);
    const uint32_t jo = a.perm[j];
    const float dw = a.dcw ? a.dcw[jo] : 1.f;
    const float *wt = a.wtab + j * 3 * kWMax;
    for (int tz = 0; tz < n[2]; tz++)
        for (int ty = 0; ty < n[1]; ty++)
            for (int tx = 0; tx < n[0]; tx++) {
                const int t[3] = {tx, ty, tz};
                int sigma[3], st[3], co[3];
                bool wrapped = false;
                for (int d = 0; d < 3; d++) {
                    const int u = lo[d] + t[d] - k.hw;
                    sigma[d] = u < 0 ? -1 : (u >= k.mos[d] ? 1 : 0);
                    co[d] = u - sigma[d] * k.mos[d];
                    st[d] = co[d] < k.hw ? 1 : (co[d] >= k.mos[d] - k.hw ? 2 : 0);
                    wrapped |= sigma[d] != 0;
                }
                if (!wrapped) continue;
                const int m = ref_fold_mult(3, st, sigma) - 1;
                if (m == 0) continue;
                float w = wt[tx] * (wt[kWMax + ty] * wt[2 * kWMax + tz]);
                if (a.sign_fold && ((co[0] + co[1] + co[2]) & 1)) w = -w;
                w *= (float)m * dw;
                const int64_t cell = (int64_t)co[2] * a.kl.s_z + (int64_t)co[1] * a.kl.s_y + co[0];
                for (int b = 0; b < a.nb; b++) {
                    float2 v;
                    if (a.layout == LAYOUT_SORTED_IL) v = samples[j * a.il_stride + b];
                    else if (a.layout == LAYOUT_SORTED) v = samples[(int64_t)b * a.Mtot + j];
                    else v = samples[(int64_t)b * a.Mtot + jo];
                    float *o = reinterpret_cast<float *>(grid + ((int64_t)b * a.F + f) * a.kl.s_bf + cell);
                    atomicAdd(o, w * v.x);
                    atomicAdd(o + 1, w * v.y);
                }
            }
}

static void launch_ref_fold_fix(const NufftPlan &p, const ConvArgs &a, const float2 *samples, float2 *grid,
                                cudaStream_t st) {
    if (!(p.flags & GB_FLAG_REFERENCE_FOLD) || p.D != 3 || p.Mtot == 0) return;
    k_ref_fold_fix<<<(unsigned)((p.Mtot + 255) / 256), 256, 0, st>>>(a, samples, grid); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

// --------------------------------------------------------------- C2NC -----

// Staged region of a home tile: tile + pad/2 cells on each side.
__host__ __device__ __forceinline__ int region_dim(const KParams &k, int d) {
    return d < k.D ? k.tile[d] + 2 * k.hw : 1;
}

// Per-warp staging area of the degridding kernel: separable weights (and
// their derivatives), region-local footprint starts and tap counts for the
// SPW samples a warp serves at once.
template <int SPW, bool GRAD>
struct DegridStage {
    float w[SPW][3][kWMax];
    float dw[GRAD ? SPW : 1][3][kWMax];
    int rs[SPW][3];
    int n[SPW][3];
};

template <int CG>
struct DegridShape {
    static constexpr int CPL = (CG >= 2) ? 2 : 1;   // coils per lane
    static constexpr int LPS = CG / CPL;            // lanes per sample
    static constexpr int SPW = 32 / LPS;            // samples per warp pass
};

// Degridding: a CTA stages its home tile plus a halo of pad/2 cells (coil
// fastest, so one sample's coil group is one contiguous row of CG complex
// values) and serves a range of the tile's home samples.  A warp serves SPW
// samples at once: LPS lanes per sample, CPL coils per lane, one 16-byte
// shared-memory load and 4 FMAs per tap per lane.
template <int CG, bool COMP, bool GRAD>
__global__ void __launch_bounds__(kThreads)
k_degrid_c2nc(ConvArgs a, const float2 *__restrict__ grid, float2 *__restrict__ out,
              const float2 *__restrict__ gweights, float *__restrict__ gout) {
    using Sh = DegridShape<CG>;
    constexpr int CPL = Sh::CPL, LPS = Sh::LPS, SPW = Sh::SPW;
    using Stage = DegridStage<SPW, GRAD>;
    extern __shared__ float4 smem_raw[];
    const KParams &k = a.k;
    const WorkItem it = a.items[blockIdx.x];
    const int grp = blockIdx.y;
    const int b0 = grp * CG;
    const int f = it.ft / k.ntiles_total;
    const int tile = it.ft - f * k.ntiles_total;
    const int tx = tile % k.ntiles[0];
    const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
    const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
    const int org[3] = {tx * k.tile[0], ty * k.tile[1], tz * k.tile[2]};
    const int R0 = region_dim(k, 0), R1 = region_dim(k, 1), R2 = region_dim(k, 2);
    const int cellsR = R0 * R1 * R2;
    const int h0 = k.D > 0 ? k.hw : 0, h1 = k.D > 1 ? k.hw : 0, h2 = k.D > 2 ? k.hw : 0;
    float2 *tile_s = reinterpret_cast<float2 *>(smem_raw);
    Stage *stages = reinterpret_cast<Stage *>(tile_s + (((size_t)cellsR * CG + 1) & ~(size_t)1));

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Stage the region, coil fastest: a warp per region row, lanes over
    // (x, coil) with coil fastest (conflict-free shared stores); the periodic
    // wrap needs one conditional per coordinate (|offset| < mos).
    {
        const int rowElems = R0 * CG;
        const int gx0 = org[0] - h0;
        for (int row = warp; row < R1 * R2; row += 8) {
            const int ry = row % R1, rz = row / R1;
            int gy = org[1] - h1 + ry;
            gy = gy < 0 ? gy + k.mos[1] : (gy >= k.mos[1] ? gy - k.mos[1] : gy);
            int gz = org[2] - h2 + rz;
            gz = gz < 0 ? gz + k.mos[2] : (gz >= k.mos[2] ? gz - k.mos[2] : gz);
            const int64_t rowoff = (int64_t)f * a.kl.s_bf + (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y;
            float2 *dst = tile_s + (size_t)row * rowElems;
            for (int e = lane; e < rowElems; e += 32) {
                const int c = e % CG;          // CG is a power of two
                const int rx = e / CG;
                int gx = gx0 + rx;
                gx = gx < 0 ? gx + k.mos[0] : (gx >= k.mos[0] ? gx - k.mos[0] : gx);
                // asynchronous 8-byte copy global -> shared (all of a thread's
                // copies in flight at once); coils beyond nb are zero-filled
                const bool in = b0 + c < a.nb;
                const float2 *src = in ? &grid[(int64_t)(b0 + c) * a.F * a.kl.s_bf + rowoff + gx] : grid;
                const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst + e);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src),
                             "r"(in ? 8 : 0)
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();

    const int sl = lane / LPS, ll = lane % LPS;
    Stage &S = stages[warp];
    const bool D3 = k.D > 2;

    for (int base = it.begin + warp * SPW; base < it.end; base += 8 * SPW) {
        // Separable weights of the warp's SPW samples, (sample, dim, tap) over lanes.
        for (int e = lane; e < SPW * 3 * kWMax; e += 32) {
            const int s = e / (3 * kWMax), d = (e / kWMax) % 3, t = e % kWMax;
            const int i = base + s;
            float w = 0.f, dw = 0.f;
            if (i < it.end && d < k.D) {
                const float sp = a.pos[(int64_t)d * a.Mtot + i] - (float)k.hw;
                const int lo = (int)ceilf(sp - k.radius);
                const int n = min((int)floorf(sp + k.radius) - lo + 1, kWMax);
                if (t < n) {
                    const int g = lo + t;
                    const float diff = sp - (float)g;
                    // tap t of the sample's table row is the weight of |diff|
                    // (both differences are exact in float)
                    w = GRAD ? kb_weight_1d(fabsf(diff), k.mos_f[d], k.one_over_W, k.beta[d], k.radius)
                             : a.wtab[((int64_t)i * k.D + d) * kWMax + t];
                    if (GRAD) {
                        dw = kb_deriv_1d(fabsf(diff), k.mos_f[d], k.one_over_W, k.beta[d], k.radius);
                        dw = (diff < 0.f) ? -dw : dw;
                    }
                    if (a.sign_fold) {
                        const float sg = sign_of(wrapmod(g, k.mos[d]));
                        w *= sg;
                        dw *= sg;
                    }
                }
                if (t == 0) {
                    const int od = d == 0 ? org[0] : (d == 1 ? org[1] : org[2]);
                    S.rs[s][d] = wrapmod(lo - od + k.hw, k.mos[d]);
                    S.n[s][d] = n;
                }
            } else if (i < it.end) {
                w = (t == 0) ? 1.f : 0.f;
                if (t == 0) { S.rs[s][d] = 0; S.n[s][d] = 1; }
            } else if (t == 0) {
                S.rs[s][d] = 0;
                S.n[s][d] = 0;
            }
            S.w[s][d][t] = w;
            if (GRAD) S.dw[s][d][t] = dw;
        }
        __syncwarp();

        const int i = base + sl;
        const int rs0 = S.rs[sl][0], rs1 = S.rs[sl][1], rs2 = S.rs[sl][2];
        const int n0 = S.n[sl][0], n1 = S.n[sl][1], n2 = S.n[sl][2];
        float wx[kWMax], dwx[GRAD ? kWMax : 1];
#pragma unroll
        for (int t = 0; t < kWMax; t++) {
            const bool in = (t < n0) && (rs0 + t < R0);
            wx[t] = in ? S.w[sl][0][t] : 0.f;
            if (GRAD) dwx[t] = in ? S.dw[sl][0][t] : 0.f;
        }
        float acc[CPL][2], cmp[COMP ? CPL : 1][2];
        float gacc[GRAD ? CPL : 1][3][2];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            acc[c][0] = acc[c][1] = 0.f;
            if (COMP) cmp[c][0] = cmp[c][1] = 0.f;
            if (GRAD)
                for (int d = 0; d < 3; d++) gacc[c][d][0] = gacc[c][d][1] = 0.f;
        }
        for (int tzi = 0; tzi < n2; tzi++) {
            const int rz = rs2 + tzi;
            if (rz >= R2) break;
            const float wz = S.w[sl][2][tzi];
            const float dwz = GRAD ? S.dw[sl][2][tzi] : 0.f;
            for (int tyi = 0; tyi < n1; tyi++) {
                const int ry = rs1 + tyi;
                if (ry >= R1) break;
                const float wy = S.w[sl][1][tyi];
                const float dwy = GRAD ? S.dw[sl][1][tyi] : 0.f;
                const float2 *row = tile_s + ((size_t)(rz * R1 + ry) * R0 + rs0) * CG + ll * CPL;
#pragma unroll
                for (int t = 0; t < kWMax; t++) {
                    if (GRAD) {
                        if (wx[t] == 0.f && dwx[t] == 0.f) continue;
                    } else if (wx[t] == 0.f) {
                        continue;
                    }
                    float2 v[CPL];
                    if (CPL == 2) {
                        const float4 q = *reinterpret_cast<const float4 *>(row + t * CG);
                        v[0] = make_float2(q.x, q.y);
                        v[CPL - 1] = make_float2(q.z, q.w);
                    } else {
                        v[0] = row[t * CG];
                    }
                    if (GRAD) {
                        const float ax = (dwx[t] * wy) * wz, ay = (wx[t] * dwy) * wz, az = (wx[t] * wy) * dwz;
#pragma unroll
                        for (int c = 0; c < CPL; c++) {
                            gacc[c][0][0] = fmaf(ax, v[c].x, gacc[c][0][0]);
                            gacc[c][0][1] = fmaf(ax, v[c].y, gacc[c][0][1]);
                            gacc[c][1][0] = fmaf(ay, v[c].x, gacc[c][1][0]);
                            gacc[c][1][1] = fmaf(ay, v[c].y, gacc[c][1][1]);
                            gacc[c][2][0] = fmaf(az, v[c].x, gacc[c][2][0]);
                            gacc[c][2][1] = fmaf(az, v[c].y, gacc[c][2][1]);
                        }
                    } else {
                        float w = wx[t] * wy;
                        if (D3) w *= wz;
#pragma unroll
                        for (int c = 0; c < CPL; c++) {
                            if (COMP) {
                                float y0 = w * v[c].x - cmp[c][0];
                                float s0 = acc[c][0] + y0;
                                cmp[c][0] = (s0 - acc[c][0]) - y0;
                                acc[c][0] = s0;
                                float y1 = w * v[c].y - cmp[c][1];
                                float s1 = acc[c][1] + y1;
                                cmp[c][1] = (s1 - acc[c][1]) - y1;
                                acc[c][1] = s1;
                            } else {
                                acc[c][0] = fmaf(w, v[c].x, acc[c][0]);
                                acc[c][1] = fmaf(w, v[c].y, acc[c][1]);
                            }
                        }
                    }
                }
            }
        }
        const bool valid = i < it.end;
        const uint32_t j = valid ? a.perm[i] : 0u;
        const int64_t idx = (a.layout != LAYOUT_ORIGINAL) ? (int64_t)i : (int64_t)j;
        if (!GRAD) {
            if (valid) {
                float scale = 1.f;
                if (a.dcw) {
                    const float dw2 = a.dcw[j];
                    scale = (a.dcw_pow == 2) ? dw2 * dw2 : dw2;
                }
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int coil = b0 + ll * CPL + c;
                    if (coil >= a.nb) break;
                    float2 val = make_float2(acc[c][0], acc[c][1]);
                    if (a.dcw) {
                        if (a.dcw_pow == 2) {
                            const float dw2 = a.dcw[j];
                            val.x = (val.x * dw2) * dw2;
                            val.y = (val.y * dw2) * dw2;
                        } else {
                            val.x *= scale;
                            val.y *= scale;
                        }
                    }
                    float2 *o = (a.layout == LAYOUT_SORTED_IL) ? out + idx * a.il_stride + coil
                                                            : out + (int64_t)coil * a.Mtot + idx;
                    if (a.accumulate) { const float2 ov = *o; val.x += ov.x; val.y += ov.y; }
                    *o = val;
                }
            }
        } else {
            float r[3] = {0.f, 0.f, 0.f};
            if (valid) {
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int coil = b0 + ll * CPL + c;
                    if (coil >= a.nb) break;
                    const float2 v = gweights[(int64_t)coil * a.Mtot + idx];
                    for (int d = 0; d < 3; d++) r[d] += v.x * gacc[c][d][0] - v.y * gacc[c][d][1];
                }
            }
#pragma unroll
            for (int off = 1; off < LPS; off <<= 1)
                for (int d = 0; d < 3; d++) r[d] += __shfl_xor_sync(0xffffffffu, r[d], off);
            if (valid && ll == 0) {
                float scale = 1.f;
                if (a.dcw) scale = (a.dcw_pow == 2) ? a.dcw[j] * a.dcw[j] : a.dcw[j];
                float *gp = gout + ((int64_t)grp * a.Mtot + j) * k.D;
                for (int d = 0; d < k.D; d++) gp[d] = r[d] * k.mos_f[d] * scale;
            }
        }
        __syncwarp();
    }
}

// Degridding, table variant (plain accumulation, no gradient): the same
// region staging and lane layout as k_degrid_c2nc, but each lane reads its
// sample's tap weights straight from the per-trajectory weight table into
// registers (no per-warp staging, no kernel evaluation) and runs a fully
// unrolled NT x NT (x NT) tap nest (unpredicated in x and y over the zero
// weights beyond the footprint; 3D slices predicated on the sample's z
// count), so the inner loop is loads and FMAs only.  NT = the largest tap count a
// footprint can have (2*ceil(W/2), plus one when W is an even integer).
// Per-sample inputs of one pass of the table degridding (loaded a pass ahead).
struct DegRaw {
    float sp[3];
    float4 t0[3], t1[3];
    uint32_t j;
    float dw;
};

template <int CG, int NT, bool D3>
__device__ __forceinline__ void degrid_table_load_raw(const ConvArgs &a, const WorkItem &it, int bs, DegRaw &r) {
    using Sh = DegridShape<CG>;
    constexpr int LPS = Sh::LPS, SPW = Sh::SPW;
    constexpr int D = D3 ? 3 : 2;
    const int lane = threadIdx.x & 31;
    const int sl = lane / LPS;
    const bool lane_ok = sl < SPW;   // false only for the 2 spare lanes of coil group 12
    const int i = bs + sl;
    const bool valid = lane_ok && i < it.end;
    const int ic = valid ? i : it.begin;   // a valid row for the loads of idle lanes
#pragma unroll
    for (int d = 0; d < D; d++) {
        r.sp[d] = a.pos[(int64_t)d * a.Mtot + ic];
        const float4 *trow = reinterpret_cast<const float4 *>(a.wtab + ((int64_t)ic * D + d) * kWMax);
        r.t0[d] = __ldg(trow);
        r.t1[d] = NT > 4 ? __ldg(trow + 1) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const bool need_j = a.layout == LAYOUT_ORIGINAL || a.dcw;
    r.j = need_j ? a.perm[ic] : (uint32_t)ic;
    r.dw = a.dcw ? a.dcw[r.j] : 1.f;
}

// The sample passes of one degridding work item over its staged region
// (tile_s: the tile plus halo, cell stride CS, zero pad after it); `cur` holds
// the first pass's inputs of this warp.
template <int CG, int NT, bool D3>
__device__ __forceinline__ void degrid_table_passes(const ConvArgs &a, const WorkItem &it, int b0, int org0,
                                                    int org1, int org2, const float2 *tile_s,
                                                    float2 *__restrict__ out, DegRaw cur) {
    using Sh = DegridShape<CG>;
    constexpr int CPL = Sh::CPL, LPS = Sh::LPS, SPW = Sh::SPW;
    constexpr int D = D3 ? 3 : 2;
    constexpr int CS = (D3 || CG == 12) ? CG : CG + 2;
    const KParams &k = a.k;
    const int R0 = region_dim(k, 0), R1 = region_dim(k, 1), R2 = region_dim(k, 2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = lane / LPS, ll = lane % LPS;
    const bool lane_ok = sl < SPW;
    DegRaw nxt;
    int base = it.begin + warp * SPW;
    for (; base < it.end; base += 8 * SPW) {
        const int i = base + sl;
        const bool valid = lane_ok && i < it.end;
        if (base + 8 * SPW < it.end) degrid_table_load_raw<CG, NT, D3>(a, it, base + 8 * SPW, nxt);
        int rs[3] = {0, 0, 0}, n[3] = {1, 1, 1};
        float w[3][NT];
#pragma unroll
        for (int d = 0; d < 3; d++) {
#pragma unroll
            for (int t = 0; t < NT; t++) w[d][t] = (t == 0) ? 1.f : 0.f;
        }
#pragma unroll
        for (int d = 0; d < D; d++) {
            const float sp = cur.sp[d] - (float)k.hw;
            const int lo = (int)ceilf(sp - k.radius);
            n[d] = valid ? min((int)floorf(sp + k.radius) - lo + 1, NT) : 0;
            const int od = d == 0 ? org0 : (d == 1 ? org1 : org2);
            int x = lo - od + k.hw;   // region-local start, |x| < 2 mos
            x = x < 0 ? x + k.mos[d] : (x >= k.mos[d] ? x - k.mos[d] : x);
            rs[d] = x;
            const int Rd = d == 0 ? R0 : (d == 1 ? R1 : R2);
            n[d] = min(n[d], Rd - x);   // the footprint lies inside the region; keep reads there
            const float tv[8] = {cur.t0[d].x, cur.t0[d].y, cur.t0[d].z, cur.t0[d].w,
                                 cur.t1[d].x, cur.t1[d].y, cur.t1[d].z, cur.t1[d].w};
            // centring checkerboard: (-1)^(cell) with cell = lo + t (mos even)
            const float s0 = (a.sign_fold && (lo & 1)) ? -1.f : 1.f;
#pragma unroll
            for (int t = 0; t < NT; t++) w[d][t] = (a.sign_fold && (t & 1)) ? -s0 * tv[t] : s0 * tv[t];
        }
        // (re, im) of each of the lane's coils, packed FP32x2 multiply-adds
        float2 acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) acc[c] = make_float2(0.f, 0.f);
        const float2 *base_s = tile_s + (((size_t)rs[2] * R1 + rs[1]) * R0 + rs[0]) * CS + ll * CPL;
        // Tap nest, unrolled to NTT taps per dimension, with no per-tap
        // predicates in x and y: the table weights beyond a footprint are zero
        // and a footprint starts at most NT-1 cells before the region's end,
        // so the extra taps read at most one row and one cell past a slice --
        // the next slice, or after the last one the zero pad.  3D slices stay
        // predicated on the sample's z count.  When every sample of the warp
        // has fewer than NT taps in every dimension (the common case when W is
        // an even integer) the NT-1 nest runs.
        auto nest = [&](auto ntc) {
            constexpr int NTT = decltype(ntc)::value;
#pragma unroll
            for (int tzi = 0; tzi < (D3 ? NTT : 1); tzi++) {
                if (tzi < n[2]) {
#pragma unroll
                    for (int tyi = 0; tyi < NTT; tyi++) {
                        {
                            const float wyz = D3 ? w[1][tyi] * w[2][tzi] : w[1][tyi];
                            const float2 *row = base_s + ((size_t)tzi * R1 + tyi) * R0 * CS;
#pragma unroll
                            for (int t = 0; t < NTT; t++) {
                                {
                                    const float wv = w[0][t] * wyz;
                                    const float2 wv2 = make_float2(wv, wv);
                                    if (CPL == 2) {
                                        const float4 q = *reinterpret_cast<const float4 *>(row + t * CS);
                                        acc[0] = __ffma2_rn(wv2, make_float2(q.x, q.y), acc[0]);
                                        acc[CPL - 1] = __ffma2_rn(wv2, make_float2(q.z, q.w), acc[CPL - 1]);
                                    } else {
                                        acc[0] = __ffma2_rn(wv2, row[t * CS], acc[0]);
                                    }
                                }
                            }
                        }
                    }
                }
            }
        };
        // only when W is an even integer can a footprint have NT = W + 1 taps
        // (an exact-integer position); otherwise NT taps are common
        const bool shorter = (NT > 4 && 2 * k.hw < NT) &&
                             __all_sync(0xffffffffu, n[0] < NT && n[1] < NT && n[2] < NT);
        if (shorter)
            nest(std::integral_constant<int, (NT > 4 ? NT - 1 : NT)>{});
        else
            nest(std::integral_constant<int, NT>{});
        if (valid) {
            const uint32_t j = cur.j;
            const int64_t idx = (a.layout != LAYOUT_ORIGINAL) ? (int64_t)i : (int64_t)j;
            const float dw = cur.dw;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                const int coil = b0 + ll * CPL + c;
                if (coil >= a.nb) break;
                float2 val = acc[c];
                if (a.dcw) {
                    if (a.dcw_pow == 2) {
                        val.x = (val.x * dw) * dw;
                        val.y = (val.y * dw) * dw;
                    } else {
                        val.x *= dw;
                        val.y *= dw;
                    }
                }
                float2 *o = (a.layout == LAYOUT_SORTED_IL) ? out + idx * a.il_stride + coil
                                                            : out + (int64_t)coil * a.Mtot + idx;
                if (a.accumulate) { const float2 ov = *o; val.x += ov.x; val.y += ov.y; }
                *o = val;
            }
        }
        cur = nxt;
    }
}

template <int CG, int NT, bool D3>
__global__ void __launch_bounds__(kThreads, D3 ? 2 : (CG == 12 ? 4 : 3))
k_degrid_table(ConvArgs a, const float2 *__restrict__ grid, float2 *__restrict__ out) {
    constexpr int SPW = DegridShape<CG>::SPW;
    // Staged cell stride in float2.  2D: padded to an odd number of 16-byte
    // chunks (conflict-free staging stores; the region copy is a large share
    // of a 2D item's work).  3D: unpadded (the copy is a few percent of an
    // item's work there and the region is large).
    constexpr int CS = (D3 || CG == 12) ? CG : CG + 2;
    static_assert(CG >= 4, "table degridding stages coil pairs");
    extern __shared__ float4 smem_raw[];
    const KParams &k = a.k;
    const WorkItem it = a.items[blockIdx.x];
    const int grp = blockIdx.y;
    const int b0 = grp * CG;
    const int f = it.ft / k.ntiles_total;
    const int tile = it.ft - f * k.ntiles_total;
    const int tx = tile % k.ntiles[0];
    const int ty = (tile / k.ntiles[0]) % k.ntiles[1];
    const int tz = tile / (k.ntiles[0] * k.ntiles[1]);
    const int org0 = tx * k.tile[0], org1 = ty * k.tile[1], org2 = tz * k.tile[2];
    const int R0 = region_dim(k, 0), R1 = region_dim(k, 1), R2 = region_dim(k, 2);
    const int h2 = D3 ? k.hw : 0;
    float2 *tile_s = reinterpret_cast<float2 *>(smem_raw);

    const int warp = threadIdx.x >> 5;

    DegRaw cur;
    int base = it.begin + warp * SPW;
    if (base < it.end) degrid_table_load_raw<CG, NT, D3>(a, it, base, cur);
    {
        // Region staging through registers.  Thread e of the CTA takes cells
        // e, e + kThreads, ... of the region in x-fastest order (every load
        // instruction is a coalesced run of one coil plane, no idle lanes at
        // row ends), loads all CG coils of UC cells before storing any (the
        // loads in flight cover the memory latency), then stores each cell's
        // coils as 16-byte chunks (with padded cells, the chunks that a warp
        // stores at once fall into different banks).
        constexpr int UC = CG <= 4 ? 2 : 1;   // cells in flight per thread
        const int ncell = R0 * R1 * R2;
        const int gx0 = org0 - k.hw, gy0 = org1 - k.hw, gz0 = org2 - h2;
        const int64_t pstride = (int64_t)a.F * a.kl.s_bf;
        const float2 *fbase = grid + (int64_t)b0 * pstride + (int64_t)f * a.kl.s_bf;
        for (int e0 = threadIdx.x; e0 < ncell; e0 += UC * kThreads) {
            float2 v[UC][CG];
#pragma unroll
            for (int u = 0; u < UC; u++) {
                const int e = e0 + u * kThreads;
                const int row = e / R0, xo = e - row * R0;
                const int rz = row / R1, ry = row - rz * R1;
                int gx = gx0 + xo, gy = gy0 + ry, gz = gz0 + rz;
                gx = gx < 0 ? gx + k.mos[0] : (gx >= k.mos[0] ? gx - k.mos[0] : gx);
                gy = gy < 0 ? gy + k.mos[1] : (gy >= k.mos[1] ? gy - k.mos[1] : gy);
                gz = gz < 0 ? gz + k.mos[2] : (gz >= k.mos[2] ? gz - k.mos[2] : gz);
                const float2 *src = fbase + (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + gx;
                const bool in = e < ncell;
#pragma unroll
                for (int c = 0; c < CG; c++)
                    v[u][c] = (in && b0 + c < a.nb) ? __ldg(src + c * pstride) : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < UC; u++) {
                const int e = e0 + u * kThreads;
                if (e < ncell) {
                    float4 *cell = reinterpret_cast<float4 *>(tile_s + (size_t)e * CS);
#pragma unroll
                    for (int q = 0; q < CG / 2; q++)
                        cell[q] = make_float4(v[u][2 * q].x, v[u][2 * q].y, v[u][2 * q + 1].x, v[u][2 * q + 1].y);
                }
            }
        }
        {
            // zero pad after the region: a tap with zero weight beyond the
            // footprint may read up to one row and one cell past it
            const int npad = (R0 + 1) * CS;
            for (int e = threadIdx.x; e < npad; e += kThreads)
                tile_s[(size_t)R0 * R1 * R2 * CS + e] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    degrid_table_passes<CG, NT, D3>(a, it, b0, org0, org1, org2, tile_s, out, cur);
}

__global__ void k_sum_groups(const float *__restrict__ part, int ngroups, int64_t n,
                             float *__restrict__ out) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float s = 0.f;
    for (int g = 0; g < ngroups; g++) s += part[(int64_t)g * n + e];
    out[e] = s;
}

// ------------------------------------------------------------ launchers ---

static ConvArgs make_args(NufftPlan &p, int nb, SampleLayout layout, const float *dcw,
                          int dcw_pow, bool sign_fold, bool accumulate) {
    ConvArgs a{};
    a.k = p.kp;
    a.pos = p.pos_sorted.get();
    a.wtab = p.wtab.get();
    a.kl = klayout_standard(p.kp);
    a.prows = p.pair_rows.get();
    a.prow_floats = p.pair_row_stride;
    a.err = p.err_flag.get();
    a.perm = p.perm.get();
    a.Mtot = p.Mtot;
    a.F = (int)p.F;
    a.nb = nb;
    a.layout = layout;
    a.il_stride = il_stride_for(nb);
    a.home_key = p.pp_key_sorted.get();
    a.dcw = dcw;
    a.dcw_pow = dcw_pow;
    a.sign_fold = sign_fold ? 1 : 0;
    a.accumulate = accumulate ? 1 : 0;
    return a;
}

static int choose_cg(int requested, int nb) {
    int cg = requested;
    if (cg != 1 && cg != 2 && cg != 4 && cg != 8 && cg != 16) cg = 8;
    while (cg > 1 && cg / 2 >= nb) cg /= 2;
    return cg;
}

// Which gridding kernel runs for a plan and batch count, with its coil group
// and the size of one CTA's partial tile (split tiles).
struct GridCfg {
    bool rows;        // k_grid_rows (else k_grid_nc2c)
    int cg;
    int rw, rpw;      // row variant: columns per lane, regions per warp
    int cpt;          // cell variant: cells per thread
    int ncg;
    int64_t part_elems;
    int smem;         // dynamic shared memory (row variant)
};

static GridCfg grid_config(const NufftPlan &p, int nb) {
    const KParams &k = p.kp;
    GridCfg c{};
    const int cells = k.tile[0] * k.tile[1] * k.tile[2];
    c.cpt = (cells + kThreads - 1) / kThreads;
    const bool comp = (p.flags & GB_FLAG_COMPENSATED) != 0;
    int cg = choose_cg(p.tiling.cg, nb);
    if (!comp && k.D >= 2 && (cg == 8 || cg == 16) && p.pair_row_stride > 0 &&
        p.pair_row_stride == pair_row_floats(k)) {
        const int rows = 64 / cg;
        const int smem = 2 * row_stage_bytes(k, cg);
        if (k.tile[1] % rows == 0 && smem <= 96 * 1024) {
            for (int rw = 4; rw <= 8 && !c.rows; rw *= 2) {
                if (k.tile[0] % rw) continue;
                const int regions = cells / (rows * rw);
                if (regions % 8) continue;
                const int rpw = regions / 8;
                if ((rpw == 1 || rpw == 2 || rpw == 4) && rpw * rw <= 16) {
                    c.rows = true;
                    c.rw = rw;
                    c.rpw = rpw;
                    c.smem = smem;
                }
            }
        }
    }
    if (!c.rows && c.cpt * cg > (comp ? 16 : 32)) cg = std::max(1, (comp ? 16 : 32) / c.cpt);
    c.cg = cg;
    c.ncg = (nb + cg - 1) / cg;
    c.part_elems = (int64_t)cg * (c.rows ? cells : kThreads * c.cpt);
    return c;
}

template <int CG, int CPT, bool COMP>
static void grid_dispatch(const ConvArgs &a, dim3 g, const float2 *s, float2 *o, cudaStream_t st) {
    k_grid_nc2c<CG, CPT, COMP><<<g, kThreads, 0, st>>>(a, s, o); ::gb::note_launch();
}

template <int CG, bool COMP>
static void grid_dispatch_cpt(int cpt, const ConvArgs &a, dim3 g, const float2 *s, float2 *o,
                              cudaStream_t st) {
    switch (cpt) {
        case 1: grid_dispatch<CG, 1, COMP>(a, g, s, o, st); break;
        case 2: grid_dispatch<CG, 2, COMP>(a, g, s, o, st); break;
        case 4: grid_dispatch<CG, 4, COMP>(a, g, s, o, st); break;
        default: fail(GB_ERR_INTERNAL, "unsupported cells per thread");
    }
}

template <int CG, int RW, int RPW, bool D3>
static void grid_rows_launch(const ConvArgs &a, dim3 g, int smem, const float2 *s, float2 *o, cudaStream_t st) {
    auto kern = k_grid_rows<CG, RW, RPW, D3>;
    if (smem > 48 * 1024)
        GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<g, kThreads, smem, st>>>(a, s, o); ::gb::note_launch();
}

template <int CG, int RW, int RPW, bool D3>
static void grid_rows_ws_launch(const ConvArgs &a, dim3 g, const float2 *s, float2 *o, cudaStream_t st) {
    auto kern = k_grid_rows_ws<CG, RW, RPW, D3>;
    const int smem = kWsStages * ws_stage_bytes(a.k, CG);
    if (smem > 48 * 1024)
        GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<g, kWsThreads, smem, st>>>(a, s, o); ::gb::note_launch();
}

template <int CG, bool D3>
static void grid_rows_ws_shape(const GridCfg &c, const ConvArgs &a, dim3 g, const float2 *s, float2 *o,
                               cudaStream_t st) {
    if (c.rw == 4 && c.rpw == 1) grid_rows_ws_launch<CG, 4, 1, D3>(a, g, s, o, st);
    else if (c.rw == 4 && c.rpw == 2) grid_rows_ws_launch<CG, 4, 2, D3>(a, g, s, o, st);
    else if (c.rw == 4 && c.rpw == 4) grid_rows_ws_launch<CG, 4, 4, D3>(a, g, s, o, st);
    else if (c.rw == 8 && c.rpw == 1) grid_rows_ws_launch<CG, 8, 1, D3>(a, g, s, o, st);
    else if (c.rw == 8 && c.rpw == 2) grid_rows_ws_launch<CG, 8, 2, D3>(a, g, s, o, st);
    else fail(GB_ERR_INTERNAL, "unsupported gridding region shape");
}

template <int CG, int RW, int RPW, bool D3>
static void grid_rows_wsp_launch(const ConvArgs &a, const float2 *s, float2 *o, cudaStream_t st) {
    auto kern = k_grid_rows_wsp<CG, RW, RPW, D3>;
    const int smem = wsp_smem_bytes(a.k, CG);
    // resident CTAs per SM for this shared-memory size (cached per instantiation)
    static int cached_smem = -1, cached_ctas = 0;
    if (smem != cached_smem) {
        GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, sms = 0, per_sm = 0;
        GB_CUDA(cudaGetDevice(&dev));
        GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWsThreads, smem));
        cached_ctas = std::max(1, per_sm) * sms;
        cached_smem = smem;
    }
    const int ctas = std::max(1, std::min(a.n_work, cached_ctas));
    kern<<<ctas, kWsThreads, smem, st>>>(a, s, o); ::gb::note_launch();
}

template <int CG, bool D3>
static void grid_rows_wsp_shape(const GridCfg &c, const ConvArgs &a, const float2 *s, float2 *o, cudaStream_t st) {
    if (c.rw == 4 && c.rpw == 1) grid_rows_wsp_launch<CG, 4, 1, D3>(a, s, o, st);
    else if (c.rw == 4 && c.rpw == 2) grid_rows_wsp_launch<CG, 4, 2, D3>(a, s, o, st);
    else if (c.rw == 4 && c.rpw == 4) grid_rows_wsp_launch<CG, 4, 4, D3>(a, s, o, st);
    else if (c.rw == 8 && c.rpw == 1) grid_rows_wsp_launch<CG, 8, 1, D3>(a, s, o, st);
    else if (c.rw == 8 && c.rpw == 2) grid_rows_wsp_launch<CG, 8, 2, D3>(a, s, o, st);
    else fail(GB_ERR_INTERNAL, "unsupported gridding region shape");
}

template <int CG, bool D3>
static void grid_rows_shape(const GridCfg &c, const ConvArgs &a, dim3 g, const float2 *s, float2 *o,
                            cudaStream_t st) {
    if (c.rw == 4 && c.rpw == 1) grid_rows_launch<CG, 4, 1, D3>(a, g, c.smem, s, o, st);
    else if (c.rw == 4 && c.rpw == 2) grid_rows_launch<CG, 4, 2, D3>(a, g, c.smem, s, o, st);
    else if (c.rw == 4 && c.rpw == 4) grid_rows_launch<CG, 4, 4, D3>(a, g, c.smem, s, o, st);
    else if (c.rw == 8 && c.rpw == 1) grid_rows_launch<CG, 8, 1, D3>(a, g, c.smem, s, o, st);
    else if (c.rw == 8 && c.rpw == 2) grid_rows_launch<CG, 8, 2, D3>(a, g, c.smem, s, o, st);
    else fail(GB_ERR_INTERNAL, "unsupported gridding region shape");
}

// How E^H E grids its own (tile-ordered) samples.
//   SCHED_ROWS: k_grid_rows on the SORTED workspace, one CTA per work item;
//   SCHED_WS:   k_grid_rows_ws on the interleaved workspace, one CTA per item;
//   SCHED_WSP:  k_grid_rows_wsp on the interleaved workspace, one persistent
//               launch over a work queue.
// The per-item warp-specialized kernel wins when the launch is a few waves
// deep: its 4-stage copy pipeline hides the staging latency that dominates a
// short launch (CG-SENSE 256^2 x 16 coils: 1082 CTAs, 1.25 -> 1.19 ms per
// recon).  On launches many waves deep the register-staged kernel's higher
// occupancy (3 CTAs of 8 warps per SM against 2 of 8 + 1) beats it (64 uneven
// frames x 12 coils: 42.0 against 45.5 ms per batch); the persistent kernel
// takes those launches.
enum GridSched { SCHED_ROWS = 0, SCHED_WS = 1, SCHED_WSP = 2 };
constexpr int kWsMaxWaves = 8;

static GridSched normal_grid_sched(const NufftPlan &p, const GridCfg &c) {
    if (!c.rows) return SCHED_ROWS;
    int sms = 0;
    GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device));
    const int64_t ctas = (int64_t)p.n_grd_items * c.ncg;
    const bool shallow = ctas <= (int64_t)kWsMaxWaves * kWsMinBlocks * sms;
    const bool wsp_fits = (int64_t)wsp_smem_bytes(p.kp, c.cg) * kWsMinBlocks <= 220 * 1024;
    switch (p.tiling.schedule) {
        case 1: return shallow ? SCHED_WS : SCHED_ROWS;
        case 2: return wsp_fits ? SCHED_WSP : (shallow ? SCHED_WS : SCHED_ROWS);
        default: return shallow ? SCHED_WS : (wsp_fits ? SCHED_WSP : SCHED_ROWS);
    }
}

// Launches the gridding kernel selected by `c` over all work items.
static void grid_dispatch_cfg(const GridCfg &c, const NufftPlan &p, const ConvArgs &a, const float2 *samples,
                              float2 *grid, cudaStream_t st) {
    dim3 g(p.n_grd_items, c.ncg);
    if (c.rows && a.layout == LAYOUT_SORTED_IL && normal_grid_sched(p, c) == SCHED_WSP) {
        const bool d3 = p.kp.D == 3;
        if (c.cg == 16) {
            if (d3) grid_rows_wsp_shape<16, true>(c, a, samples, grid, st);
            else grid_rows_wsp_shape<16, false>(c, a, samples, grid, st);
        } else {
            if (d3) grid_rows_wsp_shape<8, true>(c, a, samples, grid, st);
            else grid_rows_wsp_shape<8, false>(c, a, samples, grid, st);
        }
    } else if (c.rows && a.layout == LAYOUT_SORTED_IL) {
        const bool d3 = p.kp.D == 3;
        if (c.cg == 16) {
            if (d3) grid_rows_ws_shape<16, true>(c, a, g, samples, grid, st);
            else grid_rows_ws_shape<16, false>(c, a, g, samples, grid, st);
        } else {
            if (d3) grid_rows_ws_shape<8, true>(c, a, g, samples, grid, st);
            else grid_rows_ws_shape<8, false>(c, a, g, samples, grid, st);
        }
    } else if (c.rows) {
        const bool d3 = p.kp.D == 3;
        if (c.cg == 16) {
            if (d3) grid_rows_shape<16, true>(c, a, g, samples, grid, st);
            else grid_rows_shape<16, false>(c, a, g, samples, grid, st);
        } else {
            if (d3) grid_rows_shape<8, true>(c, a, g, samples, grid, st);
            else grid_rows_shape<8, false>(c, a, g, samples, grid, st);
        }
    } else if (p.flags & GB_FLAG_COMPENSATED) {
        switch (c.cg) {
            case 1: grid_dispatch_cpt<1, true>(c.cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, true>(c.cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, true>(c.cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, true>(c.cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, true>(c.cpt, a, g, samples, grid, st); break;
        }
    } else {
        switch (c.cg) {
            case 1: grid_dispatch_cpt<1, false>(c.cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, false>(c.cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, false>(c.cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, false>(c.cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, false>(c.cpt, a, g, samples, grid, st); break;
        }
    }
    GB_CUDA(cudaGetLastError());
}

// Allocates the split-tile counters and partial buffers for `nb` batches
// (must run outside stream capture).
void launch_grid_prepare(NufftPlan &p, int nb, cudaStream_t st) {
    const GridCfg c = grid_config(p, nb);
    if (p.grid_queue.ensure(2)) GB_CUDA(cudaMemsetAsync(p.grid_queue.get(), 0, 2 * sizeof(unsigned int), st));
    if (p.n_splits > 0) {
        const size_t need_ctr = (size_t)p.n_splits * c.ncg;
        if (p.split_counters.n < need_ctr || p.split_counter_groups == 0) {
            p.split_counters.ensure(need_ctr);
            GB_CUDA(cudaMemsetAsync(p.split_counters.get(), 0, p.split_counters.n * sizeof(unsigned int), st));
            p.split_counter_groups = c.ncg;
        }
        p.partials.ensure((size_t)p.n_slots * c.ncg * c.part_elems);
    }
}

void launch_grid(NufftPlan &p, const float2 *samples, float2 *grid, int nb, SampleLayout layout,
                 const float *dcw, bool sign_fold, bool accumulate, cudaStream_t st, const KLayout *kl) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const GridCfg c = grid_config(p, nb);
    if (layout == LAYOUT_SORTED_IL && (!c.rows || dcw))
        fail(GB_ERR_INTERNAL, "interleaved samples need the row-variant gridding kernel and no density weights");
    ConvArgs a = make_args(p, nb, layout, dcw, 1, sign_fold, accumulate);
    if (kl) a.kl = *kl;
    a.list = p.grid_list.get();
    a.items = p.grd_items.get();
    a.n_items = p.n_grd_items;
    a.splits = p.splits.get();
    a.ncg = c.ncg;
    a.part_elems = c.part_elems;
    launch_grid_prepare(p, nb, st);
    if (p.n_splits > 0) {
        a.partials = p.partials.get();
        a.counters = p.split_counters.get();
    }
    a.queue = p.grid_queue.get();
    a.n_work = p.n_grd_items * c.ncg;
    if (p.n_grd_items == 0) return;
    grid_dispatch_cfg(c, p, a, samples, grid, st);
    launch_ref_fold_fix(p, a, samples, grid, st);
}

// The sample workspace layout of E^H E follows its gridding schedule.
SampleLayout normal_op_layout(const NufftPlan &p, int nb) {
    const GridCfg c = grid_config(p, nb);
    return normal_grid_sched(p, c) == SCHED_ROWS ? LAYOUT_SORTED : LAYOUT_SORTED_IL;
}

// Scratch (split-tile partial tiles and their counters) that launch_grid
// needs for `nb` batches, in elements.
void grid_scratch_need(const NufftPlan &p, int nb, size_t *partial_elems, size_t *counter_elems) {
    const GridCfg c = grid_config(p, nb);
    *partial_elems = p.n_splits > 0 ? (size_t)p.n_slots * c.ncg * c.part_elems : 0;
    *counter_elems = p.n_splits > 0 ? (size_t)p.n_splits * c.ncg : 0;
}

// The gridding launch of launch_grid with caller-provided scratch: no device
// allocation.  `counters` must hold counter_elems zeros on entry (the kernel
// leaves them zero again when it completes).
void launch_grid_external_scratch(NufftPlan &p, const float2 *samples, float2 *grid, int nb, bool accumulate,
                                  float2 *partials, unsigned int *counters, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const GridCfg c = grid_config(p, nb);
    ConvArgs a = make_args(p, nb, LAYOUT_ORIGINAL, nullptr, 1, false, accumulate);
    a.list = p.grid_list.get();
    a.items = p.grd_items.get();
    a.n_items = p.n_grd_items;
    a.splits = p.splits.get();
    a.ncg = c.ncg;
    a.part_elems = c.part_elems;
    a.partials = partials;
    a.counters = counters;
    if (p.n_grd_items == 0) return;
    grid_dispatch_cfg(c, p, a, samples, grid, st);
    launch_ref_fold_fix(p, a, samples, grid, st);
}

template <int CG, bool GRAD>
static size_t degrid_smem_t(const KParams &k) {
    const size_t tile = (((size_t)region_dim(k, 0) * region_dim(k, 1) * region_dim(k, 2) * CG + 1) & ~(size_t)1) *
                        sizeof(float2);
    return tile + 8 * sizeof(DegridStage<DegridShape<CG>::SPW, GRAD>);
}

static size_t degrid_smem(const KParams &k, int cg, bool grad = false) {
    switch (cg) {
        case 1: return grad ? degrid_smem_t<1, true>(k) : degrid_smem_t<1, false>(k);
        case 2: return grad ? degrid_smem_t<2, true>(k) : degrid_smem_t<2, false>(k);
        case 4: return grad ? degrid_smem_t<4, true>(k) : degrid_smem_t<4, false>(k);
        case 8: return grad ? degrid_smem_t<8, true>(k) : degrid_smem_t<8, false>(k);
        default: return grad ? degrid_smem_t<16, true>(k) : degrid_smem_t<16, false>(k);
    }
}

template <int CG, bool COMP, bool GRAD>
static void degrid_launch(const ConvArgs &a, dim3 g, size_t smem, const float2 *grid, float2 *out,
                          const float2 *gw, float *gout, cudaStream_t st) {
    auto kern = k_degrid_c2nc<CG, COMP, GRAD>;
    if (smem > 48 * 1024)
        GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, kThreads, smem, st>>>(a, grid, out, gw, gout); ::gb::note_launch();
}

template <bool COMP, bool GRAD>
static void degrid_dispatch(int cg, const ConvArgs &a, dim3 g, size_t smem, const float2 *grid,
                            float2 *out, const float2 *gw, float *gout, cudaStream_t st) {
    switch (cg) {
        case 1: degrid_launch<1, COMP, GRAD>(a, g, smem, grid, out, gw, gout, st); break;
        case 2: degrid_launch<2, COMP, GRAD>(a, g, smem, grid, out, gw, gout, st); break;
        case 4: degrid_launch<4, COMP, GRAD>(a, g, smem, grid, out, gw, gout, st); break;
        case 8: degrid_launch<8, COMP, GRAD>(a, g, smem, grid, out, gw, gout, st); break;
        default: degrid_launch<16, COMP, GRAD>(a, g, smem, grid, out, gw, gout, st); break;
    }
}

static size_t degrid_table_smem(const KParams &k, int cg) {
    const int cs = (k.D == 3 || cg == 12) ? cg : cg + 2;   // cell stride of k_degrid_table
    const size_t pad = (size_t)(region_dim(k, 0) + 1) * cs;
    return ((size_t)region_dim(k, 0) * region_dim(k, 1) * region_dim(k, 2) * cs + pad) * sizeof(float2);
}

template <int CG, int NT, bool D3>
static void degrid_table_launch(const ConvArgs &a, dim3 g, size_t smem, const float2 *grid, float2 *out,
                                cudaStream_t st) {
    auto kern = k_degrid_table<CG, NT, D3>;
    if (smem > 48 * 1024)
        GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, kThreads, smem, st>>>(a, grid, out); ::gb::note_launch();
}

template <int CG, bool D3>
static void degrid_table_nt(int nt, const ConvArgs &a, dim3 g, size_t smem, const float2 *grid, float2 *out,
                            cudaStream_t st) {
    switch (nt) {
        case 4: degrid_table_launch<CG, 4, D3>(a, g, smem, grid, out, st); break;
        case 5: degrid_table_launch<CG, 5, D3>(a, g, smem, grid, out, st); break;
        case 6: degrid_table_launch<CG, 6, D3>(a, g, smem, grid, out, st); break;
        case 7: degrid_table_launch<CG, 7, D3>(a, g, smem, grid, out, st); break;
        default: degrid_table_launch<CG, 8, D3>(a, g, smem, grid, out, st); break;
    }
}

static void degrid_table_dispatch(int cg, int nt, bool d3, const ConvArgs &a, dim3 g, size_t smem,
                                  const float2 *grid, float2 *out, cudaStream_t st) {
    if (d3) {
        switch (cg) {
            case 4: degrid_table_nt<4, true>(nt, a, g, smem, grid, out, st); break;
            case 8: degrid_table_nt<8, true>(nt, a, g, smem, grid, out, st); break;
            case 12: degrid_table_nt<12, true>(nt, a, g, smem, grid, out, st); break;
            default: degrid_table_nt<16, true>(nt, a, g, smem, grid, out, st); break;
        }
    } else {
        switch (cg) {
            case 4: degrid_table_nt<4, false>(nt, a, g, smem, grid, out, st); break;
            case 8: degrid_table_nt<8, false>(nt, a, g, smem, grid, out, st); break;
            case 12: degrid_table_nt<12, false>(nt, a, g, smem, grid, out, st); break;
            default: degrid_table_nt<16, false>(nt, a, g, smem, grid, out, st); break;
        }
    }
}

static int degrid_cg(NufftPlan &p, int nb, bool grad = false) {
    int cg = choose_cg(p.tiling.cg, nb);
    while (cg > 1 && degrid_smem(p.kp, cg, grad) > 200 * 1024) cg /= 2;
    if (degrid_smem(p.kp, cg, grad) > 220 * 1024) fail(GB_ERR_INVALID_ARGUMENT, "tile too large for shared memory");
    return cg;
}

void launch_degrid(NufftPlan &p, const float2 *grid, float2 *samples, int nb, SampleLayout layout,
                   const float *dcw, int dcw_pow, bool sign_fold, bool accumulate, cudaStream_t st,
                   const KLayout *kl) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    int cg = degrid_cg(p, nb);
    // 12 coils (or a multiple of 12): one group of 12 for the table kernel
    // instead of a group of 16 with 4 empty coil slots
    const int nt12 = (int)std::floor(p.W) + 1;
    if (nb % 12 == 0 && nb % 16 != 0 && cg >= 8 && !(p.flags & GB_FLAG_COMPENSATED) && p.D >= 2 &&
        nt12 >= 4 && nt12 <= kWMax && degrid_table_smem(p.kp, 12) <= 220 * 1024)
        cg = 12;
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, layout, dcw, dcw_pow, sign_fold, accumulate);
    if (kl) a.kl = *kl;
    a.items = p.deg_items.get();
    a.n_items = p.n_deg_items;
    if (p.n_deg_items == 0) return;
    dim3 g(p.n_deg_items, ncg);
    const int nt = (int)std::floor(p.W) + 1;   // most taps a footprint can have per dimension
    if (!(p.flags & GB_FLAG_COMPENSATED) && p.D >= 2 && cg >= 4 && nt >= 4 && nt <= kWMax &&
        degrid_table_smem(p.kp, cg) <= 220 * 1024) {
        degrid_table_dispatch(cg, nt, p.D == 3, a, g, degrid_table_smem(p.kp, cg), grid, samples, st);
    } else {
        const size_t smem = degrid_smem(p.kp, cg);
        if (p.flags & GB_FLAG_COMPENSATED)
            degrid_dispatch<true, false>(cg, a, g, smem, grid, samples, nullptr, nullptr, st);
        else
            degrid_dispatch<false, false>(cg, a, g, smem, grid, samples, nullptr, nullptr, st);
    }
    GB_CUDA(cudaGetLastError());
}

void launch_traj_grad(NufftPlan &p, const float2 *grid, const float2 *weights, int nb,
                      const float *dcw, float *grad, bool sign_fold, cudaStream_t st, const KLayout *kl) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const int cg = degrid_cg(p, nb, true);
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, LAYOUT_ORIGINAL, dcw, 1, sign_fold, false);
    if (kl) a.kl = *kl;
    a.items = p.deg_items.get();
    a.n_items = p.n_deg_items;
    const int64_t n = p.Mtot * p.D;
    DevBuf<float> part;
    float *target = grad;
    if (ncg > 1) {
        part.ensure((size_t)ncg * n);
        target = part.get();
    }
    GB_CUDA(cudaMemsetAsync(target, 0, (size_t)ncg * n * sizeof(float), st));
    if (p.n_deg_items > 0) {
        dim3 g(p.n_deg_items, ncg);
        degrid_dispatch<false, true>(cg, a, g, degrid_smem(p.kp, cg, true), grid, nullptr, weights, target, st);
        GB_CUDA(cudaGetLastError());
    }
    if (ncg > 1) {
        k_sum_groups<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part.get(), ncg, n, grad); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        GB_CUDA(cudaStreamSynchronize(st));   // `part` is freed on return
    }
}

}  // namespace gb
