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
// in a different order.  Scratch: the C^2 correlation planes, twice.
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

// plane (a * nc + b) = x_b conj(x_a); grid.y = a * nc + b
__global__ void k_b1_correlation(const float2 *__restrict__ x, int nc, int64_t n, float2 *__restrict__ A) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int a = blockIdx.y / nc, b = blockIdx.y - a * nc;
    A[(int64_t)blockIdx.y * n + p] = cmulc(x[(int64_t)b * n + p], x[(int64_t)a * n + p]);
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

// Two power iterations and the coil-0 phase reference; one pixel per thread,
// the vector in registers (nc <= kB1MaxCoils).
constexpr int kB1MaxCoils = 32;

__global__ void k_b1_power(const float2 *__restrict__ A, int nc, int64_t n, float2 *__restrict__ csm) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float2 b[kB1MaxCoils], t[kB1MaxCoils];
    for (int c = 0; c < nc; c++) b[c] = make_float2(1.f, 0.f);
    for (int it = 0; it < 2; it++) {
        float nrm = 0.f;
        for (int j = 0; j < nc; j++) {
            float2 s = make_float2(0.f, 0.f);
            for (int k = 0; k < nc; k++) {
                const float2 a = A[((int64_t)k * nc + j) * n + p];
                s.x += a.x * b[k].x - a.y * b[k].y;
                s.y += a.x * b[k].y + a.y * b[k].x;
            }
            t[j] = s;
            nrm += s.x * s.x + s.y * s.y;
        }
        const float r = 1.f / sqrtf(nrm);
        for (int c = 0; c < nc; c++) b[c] = make_float2(t[c].x * r, t[c].y * r);
    }
    float sn, cs;
    sincosf(atan2f(b[0].y, b[0].x), &sn, &cs);
    for (int c = 0; c < nc; c++)   // b_c * conj(cos + i sin)
        csm[(int64_t)c * n + p] = make_float2(b[c].x * cs + b[c].y * sn, b[c].y * cs - b[c].x * sn);
}

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
    DevBuf<float2> x, A, B;
    x.ensure((size_t)nc * n);
    A.ensure((size_t)planes * n);
    B.ensure((size_t)planes * n);
    k_b1_rss_normalize<<<nblk(n), 256, 0, st>>>(images, nc, n, x.get()); note_launch();
    k_b1_correlation<<<dim3(nblk(n), planes), 256, 0, st>>>(x.get(), nc, n, A.get()); note_launch();
    float2 *src = A.get(), *dst = B.get();
    int64_t stride = 1;
    const float scale = 1.f / std::pow((float)kB1Box, (float)D);
    for (int d = 0; d < D; d++) {
        k_b1_box<<<dim3(nblk(n), planes), 256, 0, st>>>(src, dst, n, stride, len[d], d == D - 1 ? scale : 1.f);
        note_launch();
        std::swap(src, dst);
        stride *= len[d];
    }
    k_b1_power<<<nblk(n), 256, 0, st>>>(src, nc, n, csm); note_launch();
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaStreamSynchronize(st));   // scratch is freed on return
}

}  // namespace gb
