// Image-side kernels around the oversampled FFT.
//
// The reference runs, for the forward NUFFT inside the SENSE operator:
// mult_csm (sense_utilities.cu:7-18) -> pad (cuNDArray_utils.cu:273-337) ->
// deapodize (cuNFFT.cu:74-92) -> timeswitch -> cuFFT -> timeswitch -> scale
// (cuNDFFT.cpp:184-217, cuNDFFT.cu:6-36), and the mirror image for the
// adjoint ending in crop (cuNDArray_utils.cu:213-262) and
// mult_csm_conj_sum (sense_utilities.cu:66-78).  Each is a separate pass
// over the full oversampled array.
//
// Here one kernel does coil multiply + deapodization + checkerboard + 1/sqrt(G)
// and writes only the N^D interior of a padded buffer whose exterior stays
// zero (the FFT runs out of place, so the zeros are never overwritten); the
// checkerboard after the FFT is folded into the convolution weights.  On the
// way back one kernel does checkerboard + scale + deapodization + crop +
// conjugate-coil sum.
#include "gb_internal.cuh"

namespace gb {

struct ImgArgs {
    KParams k;
    const float *deap;     // [D][stride] per-dim reciprocal transforms
    int deap_stride;
    float scale;
    KLayout kl;            // layout of the oversampled array
    int full_lines;        // pad: write whole lines of the interior band (outer-major workspaces)
};

__device__ __forceinline__ void unflatten(int64_t n, const int *sz, int &x, int &y, int &z) {
    x = (int)(n % sz[0]);
    int64_t r = n / sz[0];
    y = (int)(r % sz[1]);
    z = (int)(r / sz[1]);
}

// Interior factor deap(n) * (-1)^(sum g) * scale for image pixel (x,y,z).
__device__ __forceinline__ float interior_factor(const ImgArgs &a, int x, int y, int z, int64_t &g) {
    const KParams &k = a.k;
    const int ox = (k.mos[0] - k.N[0]) >> 1, oy = (k.mos[1] - k.N[1]) >> 1, oz = (k.mos[2] - k.N[2]) >> 1;
    const int gx = x + ox, gy = y + oy, gz = z + oz;
    g = ((int64_t)gz * k.mos[1] + gy) * k.mos[0] + gx;
    float f = a.deap[x];
    if (k.D > 1) f *= a.deap[a.deap_stride + y];
    if (k.D > 2) f *= a.deap[2 * a.deap_stride + z];
    if ((gx + gy + gz) & 1) f = -f;
    return f * a.scale;
}

__device__ __forceinline__ float os_factor(const ImgArgs &a, int gx, int gy, int gz) {
    const KParams &k = a.k;
    float f = a.deap[gx];
    if (k.D > 1) f *= a.deap[a.deap_stride + gy];
    if (k.D > 2) f *= a.deap[2 * a.deap_stride + gz];
    if ((gx + gy + gz) & 1) f = -f;
    return f * a.scale;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {   // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Image rows of N0 pixels spread over a block: rpb rows per block pass,
// n0c threads per row (index math once per row, threads along x).
struct RowIter {
    int rpb, n0c, lr, x0;
};
__device__ __forceinline__ RowIter row_iter(int N0) {
    RowIter it;
    it.n0c = min(N0, (int)blockDim.x);
    it.rpb = blockDim.x / it.n0c;
    it.lr = threadIdx.x / it.n0c;
    it.x0 = threadIdx.x - it.lr * it.n0c;
    return it;
}

// Row R of the [F][N2][N1] row space -> frame, z, y.
__device__ __forceinline__ void row_coords(const KParams &k, int R, int &f, int &z, int &y, int &rem) {
    const int rpf = k.N[1] * k.N[2];
    f = R / rpf;
    rem = R - f * rpf;
    z = rem / k.N[1];
    y = rem - z * k.N[1];
}

// Forward.  csm == null: src [nb][F][NN]; else src [F][NN].  Interior only,
// or (full_lines) every padded line of the interior band -- the rows of the
// N1-row band in 2D, all mos1 rows of the N2 band slices in 3D -- with zeros
// outside the interior, so that an in-place FFT pass over the band can follow.
__global__ void k_pad_forward(ImgArgs a, const float2 *__restrict__ src, const float2 *__restrict__ csm,
                              float2 *__restrict__ dst, int nb, int F, PUpdate pu) {
    const KParams &k = a.k;
    const bool full = a.full_lines != 0;
    const int width = full ? k.mos[0] : k.N[0];
    const RowIter ri = row_iter(width);
    if (ri.lr >= ri.rpb) return;
    const int lines_y = (full && k.D == 3) ? k.mos[1] : k.N[1];   // lines per (frame, slice)
    const int lines = F * k.N[2] * lines_y;
    const int ox = (k.mos[0] - k.N[0]) >> 1, oy = (k.mos[1] - k.N[1]) >> 1, oz = (k.mos[2] - k.N[2]) >> 1;
    for (int L = blockIdx.x * ri.rpb + ri.lr; L < lines; L += gridDim.x * ri.rpb) {
        const int fz = L / lines_y, ly = L - fz * lines_y;
        const int f = fz / k.N[2], z = fz - f * k.N[2];
        const int gy = (full && k.D == 3) ? ly : ly + oy, gz = z + oz;
        const int y = gy - oy;
        const bool yin = y >= 0 && y < k.N[1];
        float fyz = a.scale;
        if (yin) {
            if (k.D > 1) fyz *= a.deap[a.deap_stride + y];
            if (k.D > 2) fyz *= a.deap[2 * a.deap_stride + z];
        }
        const int64_t gline = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y;
        const int64_t nrow = ((int64_t)z * k.N[1] + y) * k.N[0];
        for (int xw = ri.x0; xw < width; xw += ri.n0c) {
            const int gx = full ? xw : xw + ox;
            const int x = gx - ox;
            const bool in = yin && x >= 0 && x < k.N[0];
            float fac = 0.f;
            if (in) {
                fac = a.deap[x] * fyz;
                if ((gx + gy + gz) & 1) fac = -fac;
            }
            const int64_t g = gline + gx, n = nrow + x;
            if (csm) {
                float2 v = make_float2(0.f, 0.f);
                if (in) {
                    const int64_t e = (int64_t)f * k.NN + n;
                    if (pu.p) {   // p = beta p + P^2 r (segment still running), in place
                        v = pu.p[e];
                        const CgSeg &S = pu.segs[pu.seg_per_frame ? f : 0];
                        if (!S.done) {
                            const float b = (float)S.beta;
                            float2 rv = pu.r[e];
                            if (pu.P) { const float w = pu.P[e]; const float w2 = w * w; rv.x *= w2; rv.y *= w2; }
                            v = make_float2(b * v.x + rv.x, b * v.y + rv.y);
                            pu.p[e] = v;
                        }
                    } else {
                        v = src[e];
                    }
                }
#pragma unroll 8
                for (int b = 0; b < nb; b++) {
                    const float2 c = in ? cmul(v, csm[(int64_t)b * k.NN + n]) : make_float2(0.f, 0.f);
                    dst[((int64_t)b * F + f) * a.kl.s_bf + g] = make_float2(c.x * fac, c.y * fac);
                }
            } else {
#pragma unroll 4
                for (int b = 0; b < nb; b++) {
                    const float2 v = in ? src[((int64_t)b * F + f) * k.NN + n] : make_float2(0.f, 0.f);
                    dst[((int64_t)b * F + f) * a.kl.s_bf + g] = make_float2(v.x * fac, v.y * fac);
                }
            }
        }
    }
}

// Forward from an already oversampled image (full grid written).
__global__ void k_pad_forward_os(ImgArgs a, const float2 *__restrict__ src, float2 *__restrict__ dst,
                                 int64_t nbf) {
    const KParams &k = a.k;
    const int64_t total = nbf * k.G;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t bf = e / k.G, g = e - bf * k.G;
        int x, y, z;
        unflatten(g, k.mos, x, y, z);
        const float fac = os_factor(a, x, y, z);
        const float2 v = src[e];
        dst[kaddr(a.kl, bf, x, y, z)] = make_float2(v.x * fac, v.y * fac);
    }
}

// Adjoint: crop + deapodize + checkerboard + scale (+ conjugate coil sum).
__global__ void k_crop_adjoint(ImgArgs a, const float2 *__restrict__ grid, const float2 *__restrict__ csm,
                               float2 *__restrict__ dst, int nb, int F, int accumulate, float weight) {
    const KParams &k = a.k;
    const RowIter ri = row_iter(k.N[0]);
    if (ri.lr >= ri.rpb) return;
    const int rows = F * k.N[1] * k.N[2];
    const int ox = (k.mos[0] - k.N[0]) >> 1, oy = (k.mos[1] - k.N[1]) >> 1, oz = (k.mos[2] - k.N[2]) >> 1;
    for (int R = blockIdx.x * ri.rpb + ri.lr; R < rows; R += gridDim.x * ri.rpb) {
        int f, z, y, rem;
        row_coords(k, R, f, z, y, rem);
        const int gy = y + oy, gz = z + oz;
        float fyz = a.scale;
        if (k.D > 1) fyz *= a.deap[a.deap_stride + y];
        if (k.D > 2) fyz *= a.deap[2 * a.deap_stride + z];
        const int64_t grow = (int64_t)gz * a.kl.s_z + (int64_t)gy * a.kl.s_y + ox;
        const int64_t nrow = (int64_t)rem * k.N[0];
        for (int x = ri.x0; x < k.N[0]; x += ri.n0c) {
            float fac = a.deap[x] * fyz;
            if ((x + ox + gy + gz) & 1) fac = -fac;
            fac *= weight;
            const int64_t g = grow + x, n = nrow + x;
            const int64_t e = (int64_t)f * k.NN + n;
            if (csm) {
                float2 sacc = make_float2(0.f, 0.f);
#pragma unroll 8
                for (int b = 0; b < nb; b++) {
                    float2 v = grid[((int64_t)b * F + f) * a.kl.s_bf + g];
                    v = make_float2(v.x * fac, v.y * fac);
                    const float2 c = cmulc(v, csm[(int64_t)b * k.NN + n]);
                    sacc.x += c.x;
                    sacc.y += c.y;
                }
                if (accumulate) { const float2 o = dst[e]; sacc.x += o.x; sacc.y += o.y; }
                dst[e] = sacc;
            } else {
#pragma unroll 4
                for (int b = 0; b < nb; b++) {
                    const float2 v = grid[((int64_t)b * F + f) * a.kl.s_bf + g];
                    float2 r = make_float2(v.x * fac, v.y * fac);
                    float2 *o = dst + ((int64_t)b * F + f) * k.NN + n;
                    if (accumulate) { const float2 ov = *o; r.x += ov.x; r.y += ov.y; }
                    *o = r;
                }
            }
        }
    }
}

__global__ void k_crop_adjoint_os(ImgArgs a, const float2 *__restrict__ grid, float2 *__restrict__ dst,
                                  int64_t nbf, int accumulate) {
    const KParams &k = a.k;
    const int64_t total = nbf * k.G;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t bf = e / k.G, g = e - bf * k.G;
        int x, y, z;
        unflatten(g, k.mos, x, y, z);
        const float fac = os_factor(a, x, y, z);
        const float2 v = grid[kaddr(a.kl, bf, x, y, z)];
        float2 r = make_float2(v.x * fac, v.y * fac);
        if (accumulate) { const float2 o = dst[e]; r.x += o.x; r.y += o.y; }
        dst[e] = r;
    }
}

__global__ void k_timeswitch_scale(KParams k, float2 *__restrict__ data, int64_t nbf, float scale) {
    const int64_t total = nbf * k.G;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = e % k.G;
        int x, y, z;
        unflatten(g, k.mos, x, y, z);
        const float s = ((x + y + z) & 1) ? -scale : scale;
        float2 v = data[e];
        data[e] = make_float2(v.x * s, v.y * s);
    }
}

__global__ void k_deapodize_os(ImgArgs a, float2 *__restrict__ data, int64_t nbf) {
    const KParams &k = a.k;
    const int64_t total = nbf * k.G;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = e % k.G;
        int x, y, z;
        unflatten(g, k.mos, x, y, z);
        float f = a.deap[x];
        if (k.D > 1) f *= a.deap[a.deap_stride + y];
        if (k.D > 2) f *= a.deap[2 * a.deap_stride + z];
        float2 v = data[e];
        data[e] = make_float2(v.x * f, v.y * f);
    }
}

__global__ void k_multiply_dcw(const float *__restrict__ dcw, float2 *__restrict__ data, int64_t M, int nb) {
    const int64_t total = M * nb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float w = dcw[e % M];
        float2 v = data[e];
        data[e] = make_float2(v.x * w, v.y * w);
    }
}

static unsigned grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

// Blocks for the row kernels: one pass over all image rows, at most 16 per SM.
static unsigned rows_grid(int64_t rows, int width) {
    const int n0c = std::min(width, 256);
    const int64_t rpb = 256 / n0c;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows + rpb - 1) / rpb, 148 * 16));
}

static unsigned rows_grid(const NufftPlan &p) {
    return rows_grid((int64_t)p.F * p.kp.N[1] * p.kp.N[2], p.kp.N[0]);
}

static ImgArgs img_args(NufftPlan &p, bool oversampled, const KLayout *kl) {
    ImgArgs a{};
    a.k = p.kp;
    a.kl = kl ? *kl : klayout_standard(p.kp);
    a.deap = oversampled ? p.deap_os.get() : p.deap_img.get();
    a.deap_stride = oversampled ? p.maxmos : p.maxN;
    a.scale = (float)(1.0 / std::sqrt((double)p.kp.G));
    return a;
}

void launch_pad_forward(NufftPlan &p, const float2 *src, const float2 *csm, float2 *dst, int nb,
                        bool src_oversampled, cudaStream_t st, const KLayout *kl, const PUpdate *pu) {
    PUpdate pun{};
    if (pu) {
        if (!csm || src_oversampled || pu->p != src) fail(GB_ERR_INTERNAL, "direction update needs the csm pad of p");
        pun = *pu;
    }
    if (src_oversampled) {
        ImgArgs a = img_args(p, true, kl);
        const int64_t nbf = (int64_t)nb * p.F;
        k_pad_forward_os<<<grid_for(nbf * p.kp.G), 256, 0, st>>>(a, src, dst, nbf); ::gb::note_launch();
    } else {
        ImgArgs a = img_args(p, false, kl);
        // outer-major workspace under cuFFT passes: whole band lines (the
        // project-written passes read only the interior)
        a.full_lines = (kl != nullptr && p.D >= 2 && !fft_custom_ok(p)) ? 1 : 0;
        const int64_t lines = (int64_t)p.F * p.kp.N[2] * ((a.full_lines && p.D == 3) ? p.kp.mos[1] : p.kp.N[1]);
        const int width = a.full_lines ? p.kp.mos[0] : p.kp.N[0];
        k_pad_forward<<<rows_grid(lines, width), 256, 0, st>>>(a, src, csm, dst, nb, (int)p.F, pun); ::gb::note_launch();
    }
    GB_CUDA(cudaGetLastError());
}

void launch_crop_adjoint(NufftPlan &p, const float2 *grid, const float2 *csm, float2 *dst, int nb,
                         bool dst_oversampled, bool accumulate, float weight, bool fourier_deapod,
                         cudaStream_t st, const KLayout *kl) {
    (void)fourier_deapod;   // both deapodization filters have the same (real) values
    if (dst_oversampled) {
        ImgArgs a = img_args(p, true, kl);
        a.scale *= weight;
        const int64_t nbf = (int64_t)nb * p.F;
        k_crop_adjoint_os<<<grid_for(nbf * p.kp.G), 256, 0, st>>>(a, grid, dst, nbf, accumulate ? 1 : 0); ::gb::note_launch();
    } else {
        ImgArgs a = img_args(p, false, kl);
        k_crop_adjoint<<<rows_grid(p), 256, 0, st>>>(a, grid, csm, dst, nb, (int)p.F,
                                                                         accumulate ? 1 : 0, weight); ::gb::note_launch();
    }
    GB_CUDA(cudaGetLastError());
}

void launch_timeswitch_scale(NufftPlan &p, float2 *data, int nbf, float scale, cudaStream_t st) {
    k_timeswitch_scale<<<grid_for((int64_t)nbf * p.kp.G), 256, 0, st>>>(p.kp, data, nbf, scale); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

void launch_deapodize_os(NufftPlan &p, float2 *data, int nbf, cudaStream_t st) {
    ImgArgs a = img_args(p, true, nullptr);
    k_deapodize_os<<<grid_for((int64_t)nbf * p.kp.G), 256, 0, st>>>(a, data, nbf); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

void launch_multiply_dcw(const float *dcw, float2 *data, int64_t M, int nb, cudaStream_t st) {
    k_multiply_dcw<<<grid_for(M * nb), 256, 0, st>>>(dcw, data, M, nb); ::gb::note_launch();
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
