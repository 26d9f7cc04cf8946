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

#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

struct ConvArgs {
    KParams k;
    const float *pos;         // [D][Mtot] sorted positions
    const uint32_t *perm;     // sorted -> original
    const uint32_t *list;     // gridding list (sorted positions) or unused
    const WorkItem *items;
    int n_items;
    int64_t Mtot;
    int F;
    int nb;
    int layout;               // SampleLayout
    const float *dcw;         // original order, may be null
    int dcw_pow;
    int sign_fold;
    int accumulate;
    // gridding split bookkeeping
    const SplitInfo *splits;
    float2 *partials;
    unsigned int *counters;
    int ncg;
};

__device__ __forceinline__ float sign_of(int g) { return (g & 1) ? -1.f : 1.f; }

// --------------------------------------------------------------- NC2C -----

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

    __shared__ int s_a[kChunk][3];
    __shared__ int s_n[kChunk][3];
    __shared__ float s_w[kChunk][3][kWMax];
    __shared__ float2 s_v[kChunk][CG];
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

    for (int base = it.begin; base < it.end; base += kChunk) {
        const int cnt = min(kChunk, it.end - base);
        // Stage weights: one (sample, dim, tap) per thread-iteration.
        for (int e = threadIdx.x; e < kChunk * 3 * kWMax; e += kThreads) {
            const int i = e / (3 * kWMax);
            const int d = (e / kWMax) % 3;
            const int t = e % kWMax;
            float w = 0.f;
            if (i < cnt) {
                if (d < k.D) {
                    const uint32_t si = a.list[base + i];
                    const float s = a.pos[(int64_t)d * a.Mtot + si];
                    const int lo = (int)ceilf(s - k.radius);
                    const int n = (int)floorf(s + k.radius) - lo + 1;
                    if (t < n) {
                        const int p = lo + t;
                        w = kb_weight_1d(fabsf(s - (float)p), k.mos_f[d], k.one_over_W, k.beta[d], k.radius);
                        if (a.sign_fold) w *= sign_of(wrapmod(p - k.hw, k.mos[d]));
                    }
                    if (t == 0) {
                        s_a[i][d] = wrapmod(lo - k.hw - org[d], k.mos[d]);
                        s_n[i][d] = min(n, kWMax);
                    }
                } else {
                    w = (t == 0) ? 1.f : 0.f;
                    if (t == 0) { s_a[i][d] = 0; s_n[i][d] = 1; }
                }
            }
            s_w[i][d][t] = w;
        }
        // Stage values (density weights folded in).
        for (int e = threadIdx.x; e < kChunk * CG; e += kThreads) {
            const int i = e / CG, c = e % CG;
            float2 v = make_float2(0.f, 0.f);
            if (i < cnt && b0 + c < a.nb) {
                const uint32_t si = a.list[base + i];
                const uint32_t j = a.perm[si];
                const int64_t idx = (a.layout == LAYOUT_SORTED) ? (int64_t)si : (int64_t)j;
                v = samples[(int64_t)(b0 + c) * a.Mtot + idx];
                if (a.dcw) {
                    const float dw = a.dcw[j];
                    v.x = dw * v.x;
                    v.y = dw * v.y;
                }
            }
            s_v[i][c] = v;
        }
        __syncthreads();
        for (int i = 0; i < cnt; i++) {
            const int a0 = s_a[i][0], a1 = s_a[i][1], a2 = s_a[i][2];
            const int n0 = s_n[i][0], n1 = s_n[i][1], n2 = s_n[i][2];
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                int o0 = lc[c][0] - a0; if (o0 < 0) o0 += k.mos[0];
                int o1 = lc[c][1] - a1; if (o1 < 0) o1 += k.mos[1];
                int o2 = lc[c][2] - a2; if (o2 < 0) o2 += k.mos[2];
                if (o0 < n0 && o1 < n1 && o2 < n2) {
                    const float w = (s_w[i][0][o0] * s_w[i][1][o1]) * s_w[i][2][o2];
#pragma unroll
                    for (int q = 0; q < CG; q++) {
                        const float2 v = s_v[i][q];
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
        __syncthreads();
    }

    const int64_t G = k.G;
    bool cell_ok[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++)
        cell_ok[c] = lc[c][0] < k.tile[0] && lc[c][1] < k.tile[1] && lc[c][2] < k.tile[2];
    auto cell_index = [&](int c) -> int64_t {
        const int gx = org[0] + lc[c][0], gy = org[1] + lc[c][1], gz = org[2] + lc[c][2];
        return ((int64_t)gz * k.mos[1] + gy) * k.mos[0] + gx;
    };
    if (it.split < 0) {
#pragma unroll
        for (int c = 0; c < CPT; c++) {
            if (!cell_ok[c]) continue;
            const int64_t g = cell_index(c);
#pragma unroll
            for (int q = 0; q < CG; q++) {
                if (b0 + q >= a.nb) break;
                float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * G + g;
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
            float2 *o = grid + ((int64_t)(b0 + q) * a.F + f) * G + g;
            float2 v = make_float2(sr, sim);
            if (a.accumulate) { float2 old = *o; v.x += old.x; v.y += old.y; }
            *o = v;
        }
    }
}

// --------------------------------------------------------------- C2NC -----

// Staged region of a home tile: tile + pad/2 cells on each side.
__host__ __device__ __forceinline__ int region_dim(const KParams &k, int d) {
    return d < k.D ? k.tile[d] + 2 * k.hw : 1;
}

template <int CG, bool COMP, bool GRAD>
__global__ void __launch_bounds__(kThreads)
k_degrid_c2nc(ConvArgs a, const float2 *__restrict__ grid, float2 *__restrict__ out,
              const float2 *__restrict__ gweights, float *__restrict__ gout) {
    extern __shared__ float4 smem_raw[];
    float2 *tile_s = reinterpret_cast<float2 *>(smem_raw);
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

    // Stage the region, coil fastest.
    for (int e = threadIdx.x; e < cellsR * CG; e += kThreads) {
        const int c = e % CG;
        const int cell = e / CG;
        const int rx = cell % R0, ry = (cell / R0) % R1, rz = cell / (R0 * R1);
        const int gx = wrapmod(org[0] - h0 + rx, k.mos[0]);
        const int gy = wrapmod(org[1] - h1 + ry, k.mos[1]);
        const int gz = wrapmod(org[2] - h2 + rz, k.mos[2]);
        float2 v = make_float2(0.f, 0.f);
        if (b0 + c < a.nb)
            v = __ldg(&grid[((int64_t)(b0 + c) * a.F + f) * k.G + ((int64_t)gz * k.mos[1] + gy) * k.mos[0] + gx]);
        tile_s[e] = v;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int LPS = 2 * CG;              // lanes per slot (coil x re/im)
    constexpr int NS = 32 / LPS;             // slots: split of the y taps
    const int slot = lane / LPS;
    const int cl = lane % LPS;               // coil*2 + comp
    const float *tile_f = reinterpret_cast<const float *>(tile_s);

    for (int i = it.begin + warp; i < it.end; i += 8) {
        // Lanes 0..23 compute the (dim, tap) weights.
        const int wd = lane / kWMax, wt = lane % kWMax;
        float w = 0.f, dw = 0.f;
        int lo = 0, n = 1;
        float sp = 0.f;
        if (wd < k.D) {
            sp = a.pos[(int64_t)wd * a.Mtot + i] - (float)k.hw;
            lo = (int)ceilf(sp - k.radius);
            n = min((int)floorf(sp + k.radius) - lo + 1, kWMax);
            if (wt < n) {
                const int g = lo + wt;
                const float diff = sp - (float)g;
                w = kb_weight_1d(fabsf(diff), k.mos_f[wd], k.one_over_W, k.beta[wd], k.radius);
                if (GRAD) {
                    dw = kb_deriv_1d(fabsf(diff), k.mos_f[wd], k.one_over_W, k.beta[wd], k.radius);
                    dw = (diff < 0.f) ? -dw : dw;
                }
                if (a.sign_fold) {
                    const float sg = sign_of(wrapmod(g, k.mos[wd]));
                    w *= sg;
                    dw *= sg;
                }
            }
        } else if (wd < 3) {
            w = (wt == 0) ? 1.f : 0.f;
        }
        // Region-local start of the footprint per dim and tap counts.
        int rs[3], nn[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const int lo_d = __shfl_sync(0xffffffffu, lo, d * kWMax);
            const int n_d = __shfl_sync(0xffffffffu, n, d * kWMax);
            if (d < k.D) {
                rs[d] = wrapmod(lo_d - org[d] + k.hw, k.mos[d]);
                nn[d] = n_d;
            } else {
                rs[d] = 0;
                nn[d] = 1;
            }
        }
        float wx[kWMax], dwx[kWMax];
#pragma unroll
        for (int t = 0; t < kWMax; t++) {
            wx[t] = __shfl_sync(0xffffffffu, w, t);
            if (GRAD) dwx[t] = __shfl_sync(0xffffffffu, dw, t);
            // taps outside the staged region carry zero weight (see header)
            if (t >= nn[0] || rs[0] + t >= R0) { wx[t] = 0.f; if (GRAD) dwx[t] = 0.f; }
        }
        float acc = 0.f, cmp = 0.f;
        float gx_acc = 0.f, gy_acc = 0.f, gz_acc = 0.f;
        for (int tzi = 0; tzi < nn[2]; tzi++) {
            const float wz = __shfl_sync(0xffffffffu, w, 2 * kWMax + tzi);
            const float dwz = GRAD ? __shfl_sync(0xffffffffu, dw, 2 * kWMax + tzi) : 0.f;
            const int rz = rs[2] + tzi;
            for (int tyi = 0; tyi < nn[1]; tyi++) {
                const float wy = __shfl_sync(0xffffffffu, w, kWMax + tyi);
                const float dwy = GRAD ? __shfl_sync(0xffffffffu, dw, kWMax + tyi) : 0.f;
                const int ry = rs[1] + tyi;
                if ((tyi % NS) != slot || ry >= R1 || rz >= R2) continue;
                const float *row = tile_f + ((int64_t)(rz * R1 + ry) * R0 + rs[0]) * LPS + cl;
                if (GRAD) {
#pragma unroll
                    for (int t = 0; t < kWMax; t++) {
                        const float gv = (wx[t] != 0.f || dwx[t] != 0.f) ? row[t * LPS] : 0.f;
                        gx_acc = fmaf(dwx[t] * wy * wz, gv, gx_acc);
                        gy_acc = fmaf(wx[t] * dwy * wz, gv, gy_acc);
                        gz_acc = fmaf(wx[t] * wy * dwz, gv, gz_acc);
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < kWMax; t++) {
                        if (wx[t] != 0.f) {
                            const float wt2 = (wx[t] * wy) * wz;
                            const float gv = row[t * LPS];
                            if (COMP) {
                                float y = wt2 * gv - cmp;
                                float tt = acc + y;
                                cmp = (tt - acc) - y;
                                acc = tt;
                            } else {
                                acc = fmaf(wt2, gv, acc);
                            }
                        }
                    }
                }
            }
        }
        const uint32_t j = a.perm[i];
        if (!GRAD) {
            if (COMP) acc -= cmp;
#pragma unroll
            for (int off = LPS; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
            const int coil = b0 + (cl >> 1);
            if (slot == 0 && coil < a.nb) {
                float val = acc;
                if (a.dcw) {
                    const float dw2 = a.dcw[j];
                    val = (a.dcw_pow == 2) ? (val * dw2) * dw2 : val * dw2;
                }
                const int64_t idx = (a.layout == LAYOUT_SORTED) ? (int64_t)i : (int64_t)j;
                float *o = reinterpret_cast<float *>(out + (int64_t)coil * a.Mtot + idx) + (cl & 1);
                if (a.accumulate) val += *o;
                *o = val;
            }
        } else {
            // sum_coil Re(v * g):  lane (c, re) contributes v.re*g.re,
            // lane (c, im) contributes -v.im*g.im.
            const int coil = b0 + (cl >> 1);
            float vcomp = 0.f;
            if (coil < a.nb) {
                const int64_t idx = (a.layout == LAYOUT_SORTED) ? (int64_t)i : (int64_t)j;
                const float2 v = gweights[(int64_t)coil * a.Mtot + idx];
                vcomp = (cl & 1) ? -v.y : v.x;
            }
            float r0 = vcomp * gx_acc, r1 = vcomp * gy_acc, r2 = vcomp * gz_acc;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                r0 += __shfl_xor_sync(0xffffffffu, r0, off);
                r1 += __shfl_xor_sync(0xffffffffu, r1, off);
                r2 += __shfl_xor_sync(0xffffffffu, r2, off);
            }
            if (lane == 0) {
                float scale = 1.f;
                if (a.dcw) scale = (a.dcw_pow == 2) ? a.dcw[j] * a.dcw[j] : a.dcw[j];
                float *g = gout + ((int64_t)grp * a.Mtot + j) * k.D;
                const float r[3] = {r0, r1, r2};
                for (int d = 0; d < k.D; d++) g[d] = r[d] * k.mos_f[d] * scale;
            }
        }
    }
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
    a.perm = p.perm.get();
    a.Mtot = p.Mtot;
    a.F = (int)p.F;
    a.nb = nb;
    a.layout = layout;
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

static int grid_cg(NufftPlan &p, int nb, int cpt, bool comp) {
    int cg = choose_cg(p.tiling.cg, nb);
    if (cpt * cg > (comp ? 16 : 32)) cg = std::max(1, (comp ? 16 : 32) / cpt);
    return cg;
}

// Allocates the split-tile counters and partial buffers for `nb` batches
// (must run outside stream capture).
void launch_grid_prepare(NufftPlan &p, int nb, cudaStream_t st) {
    const KParams &k = p.kp;
    const int cpt = (k.tile[0] * k.tile[1] * k.tile[2] + kThreads - 1) / kThreads;
    const int cells = kThreads * cpt;
    const bool comp = (p.flags & GB_FLAG_COMPENSATED) != 0;
    const int cg = grid_cg(p, nb, cpt, comp);
    const int ncg = (nb + cg - 1) / cg;
    if (p.n_splits > 0) {
        const size_t need_ctr = (size_t)p.n_splits * ncg;
        if (p.split_counters.n < need_ctr || p.split_counter_groups == 0) {
            p.split_counters.ensure(need_ctr);
            GB_CUDA(cudaMemsetAsync(p.split_counters.get(), 0, p.split_counters.n * sizeof(unsigned int), st));
            p.split_counter_groups = ncg;
        }
        p.partials.ensure((size_t)p.n_slots * ncg * cg * cells);
    }
}

void launch_grid(NufftPlan &p, const float2 *samples, float2 *grid, int nb, SampleLayout layout,
                 const float *dcw, bool sign_fold, bool accumulate, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const KParams &k = p.kp;
    const int cells = k.tile[0] * k.tile[1] * k.tile[2];
    const int cpt = (cells + kThreads - 1) / kThreads;
    const bool comp = (p.flags & GB_FLAG_COMPENSATED) != 0;
    const int cg = grid_cg(p, nb, cpt, comp);
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, layout, dcw, 1, sign_fold, accumulate);
    a.list = p.grid_list.get();
    a.items = p.grd_items.get();
    a.n_items = p.n_grd_items;
    a.splits = p.splits.get();
    a.ncg = ncg;
    if (p.n_splits > 0) {
        launch_grid_prepare(p, nb, st);
        a.partials = p.partials.get();
        a.counters = p.split_counters.get();
    }
    if (p.n_grd_items == 0) return;
    dim3 g(p.n_grd_items, ncg);
    if (comp) {
        switch (cg) {
            case 1: grid_dispatch_cpt<1, true>(cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, true>(cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, true>(cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, true>(cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, true>(cpt, a, g, samples, grid, st); break;
        }
    } else {
        switch (cg) {
            case 1: grid_dispatch_cpt<1, false>(cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, false>(cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, false>(cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, false>(cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, false>(cpt, a, g, samples, grid, st); break;
        }
    }
    GB_CUDA(cudaGetLastError());
}

// Scratch (split-tile partial tiles and their counters) that launch_grid
// needs for `nb` batches, in elements.
void grid_scratch_need(const NufftPlan &p, int nb, size_t *partial_elems, size_t *counter_elems) {
    const KParams &k = p.kp;
    const int cpt = (k.tile[0] * k.tile[1] * k.tile[2] + kThreads - 1) / kThreads;
    const bool comp = (p.flags & GB_FLAG_COMPENSATED) != 0;
    int cg = choose_cg(p.tiling.cg, nb);
    if (cpt * cg > (comp ? 16 : 32)) cg = std::max(1, (comp ? 16 : 32) / cpt);
    const int ncg = (nb + cg - 1) / cg;
    *partial_elems = p.n_splits > 0 ? (size_t)p.n_slots * ncg * cg * kThreads * cpt : 0;
    *counter_elems = p.n_splits > 0 ? (size_t)p.n_splits * ncg : 0;
}

// The gridding launch of launch_grid with caller-provided scratch: no device
// allocation.  `counters` must hold counter_elems zeros on entry (the kernel
// leaves them zero again when it completes).
void launch_grid_external_scratch(NufftPlan &p, const float2 *samples, float2 *grid, int nb, bool accumulate,
                                  float2 *partials, unsigned int *counters, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const KParams &k = p.kp;
    const int cpt = (k.tile[0] * k.tile[1] * k.tile[2] + kThreads - 1) / kThreads;
    const bool comp = (p.flags & GB_FLAG_COMPENSATED) != 0;
    const int cg = grid_cg(p, nb, cpt, comp);
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, LAYOUT_ORIGINAL, nullptr, 1, false, accumulate);
    a.list = p.grid_list.get();
    a.items = p.grd_items.get();
    a.n_items = p.n_grd_items;
    a.splits = p.splits.get();
    a.ncg = ncg;
    a.partials = partials;
    a.counters = counters;
    if (p.n_grd_items == 0) return;
    dim3 g(p.n_grd_items, ncg);
    if (comp) {
        switch (cg) {
            case 1: grid_dispatch_cpt<1, true>(cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, true>(cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, true>(cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, true>(cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, true>(cpt, a, g, samples, grid, st); break;
        }
    } else {
        switch (cg) {
            case 1: grid_dispatch_cpt<1, false>(cpt, a, g, samples, grid, st); break;
            case 2: grid_dispatch_cpt<2, false>(cpt, a, g, samples, grid, st); break;
            case 4: grid_dispatch_cpt<4, false>(cpt, a, g, samples, grid, st); break;
            case 8: grid_dispatch_cpt<8, false>(cpt, a, g, samples, grid, st); break;
            default: grid_dispatch_cpt<16, false>(cpt, a, g, samples, grid, st); break;
        }
    }
    GB_CUDA(cudaGetLastError());
}

static size_t degrid_smem(const KParams &k, int cg) {
    return (size_t)region_dim(k, 0) * region_dim(k, 1) * region_dim(k, 2) * cg * sizeof(float2);
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

static int degrid_cg(NufftPlan &p, int nb) {
    int cg = choose_cg(p.tiling.cg, nb);
    while (cg > 1 && degrid_smem(p.kp, cg) > 200 * 1024) cg /= 2;
    if (degrid_smem(p.kp, cg) > 220 * 1024) fail(GB_ERR_INVALID_ARGUMENT, "tile too large for shared memory");
    return cg;
}

void launch_degrid(NufftPlan &p, const float2 *grid, float2 *samples, int nb, SampleLayout layout,
                   const float *dcw, int dcw_pow, bool sign_fold, bool accumulate, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const int cg = degrid_cg(p, nb);
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, layout, dcw, dcw_pow, sign_fold, accumulate);
    a.items = p.deg_items.get();
    a.n_items = p.n_deg_items;
    if (p.n_deg_items == 0) return;
    dim3 g(p.n_deg_items, ncg);
    const size_t smem = degrid_smem(p.kp, cg);
    if (p.flags & GB_FLAG_COMPENSATED)
        degrid_dispatch<true, false>(cg, a, g, smem, grid, samples, nullptr, nullptr, st);
    else
        degrid_dispatch<false, false>(cg, a, g, smem, grid, samples, nullptr, nullptr, st);
    GB_CUDA(cudaGetLastError());
}

void launch_traj_grad(NufftPlan &p, const float2 *grid, const float2 *weights, int nb,
                      const float *dcw, float *grad, bool sign_fold, cudaStream_t st) {
    if (!p.prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
    const int cg = degrid_cg(p, nb);
    const int ncg = (nb + cg - 1) / cg;
    ConvArgs a = make_args(p, nb, LAYOUT_ORIGINAL, dcw, 1, sign_fold, false);
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
        degrid_dispatch<false, true>(cg, a, g, degrid_smem(p.kp, cg), grid, nullptr, weights, target, st);
        GB_CUDA(cudaGetLastError());
    }
    if (ncg > 1) {
        k_sum_groups<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part.get(), ncg, n, grad); ::gb::note_launch();
        GB_CUDA(cudaGetLastError());
        GB_CUDA(cudaStreamSynchronize(st));   // `part` is freed on return
    }
}

}  // namespace gb
