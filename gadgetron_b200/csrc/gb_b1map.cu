// Coil sensitivity (b1) map estimation from coil images (estimate_b1_map,
// toolboxes/mri/pmri/gpu/b1_map.cu:29-118):
//   1. keep the first target_coils coil images and divide each pixel by the
//      root-sum-of-squares over those coils (:77-78, :128-168);
//   2. per pixel, the coil correlation matrix A[a][b] = x_b conj(x_a)
//      (:170-217);
//   3. smooth every entry of A over a 7^D box around the pixel, cells outside
//      the image counted as zero, scaled by 1 / 7^D (:219-636);
//   4. per pixel, two power iterations from b = (1, ..., 1):
//      t_j = sum_k A[k][j] b_k, b = t / ||t|| (:646-746);
//   5. rotate every pixel's vector so that coil 0 is real and non-negative:
//      b_c *= exp(-i arg b_0) (:775-808).
// The box is applied as separable passes (x, then y, then z), the same sums
// in a different order; the correlation products are formed inside the x
// pass, so the unsmoothed planes never reach memory.  Scratch: the
// normalised coil images and the C^2 correlation planes twice, kept per
// device between calls (grown to the largest call, never shrunk) so that a
// pipeline re-estimating the map every frame allocates nothing.
#include <cmath>

#include "gb_internal.cuh"

namespace gb {

namespace {

constexpr int kB1Box = 7;   // box width of the smoothing (b1_map.cu:19)

__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {   // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

__global__ void k_b1_rss_normalize(const float2 *__restrict__ in, int nc, int64_t n, float2 *__restrict__ out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float rss = 0.f;
    for (int c = 0; c < nc; c++) {
        const float2 v = in[(int64_t)c * n + p];
        rss += v.x * v.x + v.y * v.y;
    }
    const float r = 1.f / sqrtf(rss);
    for (int c = 0; c < nc; c++) {
        const float2 v = in[(int64_t)c * n + p];
        out[(int64_t)c * n + p] = make_float2(v.x * r, v.y * r);
    }
}

// Correlation and its box sum along x in one pass: plane (a * nc + b) at
// pixel p = sum over the kB1Box x-neighbours q of p inside the image of
// x_b(q) conj(x_a(q)); grid.y = a * nc + b.  `scale` is applied when x is
// the last smoothed dimension.
__global__ void k_b1_corr_box_x(const float2 *__restrict__ x, int nc, int64_t n, int len0, float scale,
                                float2 *__restrict__ A) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int a = blockIdx.y / nc, b = blockIdx.y - a * nc;
    const float2 *xa = x + (int64_t)a * n, *xb = x + (int64_t)b * n;
    const int pos = (int)(p % len0);
    float2 s = make_float2(0.f, 0.f);
    for (int k = -(kB1Box >> 1); k <= (kB1Box >> 1); k++) {
        const int q = pos + k;
        if (q < 0 || q >= len0) continue;
        const float2 v = cmulc(xb[p + k], xa[p + k]);
        s.x += v.x;
        s.y += v.y;
    }
    A[(int64_t)blockIdx.y * n + p] = make_float2(s.x * scale, s.y * scale);
}

// 2D: correlation products of a TX x TY pixel tile plus a 3-cell halo in
// shared memory (zero outside the image), the x pass, then the y pass and the
// 1 / 7^2 scale, one plane per blockIdx.y -- the sums and their order are
// those of k_b1_corr_box_x followed by k_b1_box, without the intermediate
// planes in memory.
constexpr int kB1TX = 32, kB1TY = 16, kB1H = kB1Box >> 1;

__global__ void __launch_bounds__(256) k_b1_corr_box_xy(const float2 *__restrict__ x, int nc, int nx, int ny,
                                                        int tiles_x, float scale, float2 *__restrict__ A) {
    constexpr int PW = kB1TX + 2 * kB1H, PH = kB1TY + 2 * kB1H;
    __shared__ float2 P[PH][PW];       // products, halo included
    __shared__ float2 Q[PH][kB1TX];    // x-pass sums
    const int64_t n = (int64_t)nx * ny;
    const int a = blockIdx.y / nc, b = blockIdx.y - a * nc;
    const float2 *xa = x + (int64_t)a * n, *xb = x + (int64_t)b * n;
    const int tx0 = (blockIdx.x % tiles_x) * kB1TX, ty0 = (blockIdx.x / tiles_x) * kB1TY;
    for (int e = threadIdx.x; e < PH * PW; e += blockDim.x) {
        const int py = e / PW, px = e - py * PW;
        const int gx = tx0 + px - kB1H, gy = ty0 + py - kB1H;
        float2 v = make_float2(0.f, 0.f);
        if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
            const int64_t g = (int64_t)gy * nx + gx;
            v = cmulc(xb[g], xa[g]);
        }
        P[py][px] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < PH * kB1TX; e += blockDim.x) {
        const int py = e / kB1TX, qx = e - py * kB1TX;
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kB1Box; k++) {
            const float2 v = P[py][qx + k];
            s.x += v.x;
            s.y += v.y;
        }
        Q[py][qx] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kB1TY * kB1TX; e += blockDim.x) {
        const int oy = e / kB1TX, ox = e - oy * kB1TX;
        const int gx = tx0 + ox, gy = ty0 + oy;
        if (gx >= nx || gy >= ny) continue;
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kB1Box; k++) {
            const float2 v = Q[oy + k][ox];
            s.x += v.x;
            s.y += v.y;
        }
        A[(int64_t)blockIdx.y * n + (int64_t)gy * nx + gx] = make_float2(s.x * scale, s.y * scale);
    }
}

// Box sum of width kB1Box along one dimension (stride between neighbours
// `stride`, extent `len`, zero outside), every plane; the last pass scales.
__global__ void k_b1_box(const float2 *__restrict__ in, float2 *__restrict__ out, int64_t n, int64_t stride,
                         int len, float scale) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int64_t plane = (int64_t)blockIdx.y * n;
    const int pos = (int)((p / stride) % len);
    float2 s = make_float2(0.f, 0.f);
    for (int k = -(kB1Box >> 1); k <= (kB1Box >> 1); k++) {
        const int q = pos + k;
        if (q < 0 || q >= len) continue;
        const float2 v = in[plane + p + (int64_t)k * stride];
        s.x += v.x;
        s.y += v.y;
    }
    out[plane + p] = make_float2(s.x * scale, s.y * scale);
}

// Two power iterations and the coil-0 phase reference; one pixel per thread.
// NCB bounds the coil count at compile time so that the vectors stay in
// registers (loops fully unrolled, coils >= nc predicated off).
constexpr int kB1MaxCoils = 32;

template <int NCB>
__global__ void __launch_bounds__(256, NCB <= 16 ? 2 : 1) k_b1_power(const float2 *__restrict__ A, int nc, int64_t n, float2 *__restrict__ csm) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float2 b[NCB], t[NCB];
#pragma unroll
    for (int c = 0; c < NCB; c++) b[c] = make_float2(c < nc ? 1.f : 0.f, 0.f);
    for (int it = 0; it < 2; it++) {
        float nrm = 0.f;
#pragma unroll
        for (int j = 0; j < NCB; j++) {
            float2 s = make_float2(0.f, 0.f);
            if (j < nc) {
#pragma unroll
                for (int k = 0; k < NCB; k++) {
                    if (k < nc) {
                        const float2 a = A[((int64_t)k * nc + j) * n + p];
                        s.x += a.x * b[k].x - a.y * b[k].y;
                        s.y += a.x * b[k].y + a.y * b[k].x;
                    }
                }
                nrm += s.x * s.x + s.y * s.y;
            }
            t[j] = s;
        }
        const float r = 1.f / sqrtf(nrm);
#pragma unroll
        for (int c = 0; c < NCB; c++) b[c] = make_float2(t[c].x * r, t[c].y * r);
    }
    float sn, cs;
    sincosf(atan2f(b[0].y, b[0].x), &sn, &cs);
#pragma unroll
    for (int c = 0; c < NCB; c++)   // b_c * conj(cos + i sin)
        if (c < nc) csm[(int64_t)c * n + p] = make_float2(b[c].x * cs + b[c].y * sn, b[c].y * cs - b[c].x * sn);
}

// Scratch kept per device between calls; the mutex is held for a whole call.
struct B1Scratch {
    std::mutex mu;
    DevBuf<float2> x, A, B;
};

unsigned int nblk(int64_t n) { return (unsigned int)((n + 255) / 256); }

}  // namespace

void estimate_b1_map(int D, const uint64_t *dims, int ncoils, int target_coils, const float2 *images, float2 *csm,
                     cudaStream_t st) {
    if (D < 1 || D > 3 || !dims || !images || !csm || ncoils <= 0)
        fail(GB_ERR_INVALID_ARGUMENT, "estimate_b1_map:: dimensionality mismatch.");
    const int nc = (target_coils <= 0 || target_coils > ncoils) ? ncoils : target_coils;
    if (nc > kB1MaxCoils) fail(GB_ERR_INVALID_ARGUMENT, "estimate_b1_map: at most 32 target coils are supported");
    int64_t n = 1;
    int len[3] = {1, 1, 1};
    for (int d = 0; d < D; d++) {
        if (dims[d] == 0 || dims[d] > (1u << 20)) fail(GB_ERR_INVALID_ARGUMENT, "estimate_b1_map: invalid image size");
        len[d] = (int)dims[d];
        n *= (int64_t)dims[d];
    }
    const int planes = nc * nc;
    if ((int64_t)planes * n > ((int64_t)1 << 31)) fail(GB_ERR_INVALID_ARGUMENT, "estimate_b1_map: images too large");
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    B1Scratch &sc = device_scratch<B1Scratch>(dev);
    std::lock_guard<std::mutex> lock(sc.mu);
    sc.x.ensure((size_t)nc * n);
    sc.A.ensure((size_t)planes * n);
    if (D > 2) sc.B.ensure((size_t)planes * n);
    const float scale = 1.f / std::pow((float)kB1Box, (float)D);
    k_b1_rss_normalize<<<nblk(n), 256, 0, st>>>(images, nc, n, sc.x.get()); note_launch();
    float2 *src = sc.A.get(), *dst = sc.B.get();
    int64_t stride = len[0];
    int d = 1;
    if (D == 2) {   // both passes on shared-memory tiles
        const int tiles_x = (len[0] + kB1TX - 1) / kB1TX, tiles_y = (len[1] + kB1TY - 1) / kB1TY;
        k_b1_corr_box_xy<<<dim3((unsigned)(tiles_x * tiles_y), planes), 256, 0, st>>>(
            sc.x.get(), nc, len[0], len[1], tiles_x, scale, sc.A.get());
        note_launch();
        d = D;
    } else {
        k_b1_corr_box_x<<<dim3(nblk(n), planes), 256, 0, st>>>(sc.x.get(), nc, n, len[0], D == 1 ? scale : 1.f,
                                                                sc.A.get());
        note_launch();
    }
    for (; d < D; d++) {
        k_b1_box<<<dim3(nblk(n), planes), 256, 0, st>>>(src, dst, n, stride, len[d], d == D - 1 ? scale : 1.f);
        note_launch();
        std::swap(src, dst);
        stride *= len[d];
    }
    if (nc <= 4)
        k_b1_power<4><<<nblk(n), 256, 0, st>>>(src, nc, n, csm);
    else if (nc <= 8)
        k_b1_power<8><<<nblk(n), 256, 0, st>>>(src, nc, n, csm);
    else if (nc <= 16)
        k_b1_power<16><<<nblk(n), 256, 0, st>>>(src, nc, n, csm);
    else
        k_b1_power<32><<<nblk(n), 256, 0, st>>>(src, nc, n, csm);
    note_launch();
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaStreamSynchronize(st));   // the scratch is free for the next call on return
}

}  // namespace gb
