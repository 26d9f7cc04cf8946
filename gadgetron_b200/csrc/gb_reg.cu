// Image regulariser and SENSE preconditioner weights (setup once per
// reconstruction, outside the CG loop).
//
// imageOperator::compute (toolboxes/operators/imageOperator.h:27-45) with the
// offset estimate of cuImageOperator (toolboxes/operators/gpu/cuImageOperator.h:35-62):
//   scale = n / asum(reg), asum = sum |re| + |im|;
//   a_i = |scale * reg_i|;
//   offset = (k + 1) * max(a) / 50000, k the first bin of the 50000-bin
//            histogram of a / max(a) at which the cumulative count reaches
//            1% of n (only with offset estimation);
//   image_i = 1 / (a_i + offset).
// Every float operation is rounded as written (no contraction), so the bins
// and the image match a float restatement of the same formulas; asum is
// summed in FP64 and rounded once.
//
// Preconditioner weights of gpuCgSenseGadget.cpp:167-176:
//   w = 1 / sqrt(sum_c |csm_c|^2 + kappa * image).
#include <vector>

#include "gb_internal.cuh"

namespace gb {

namespace {

constexpr int kHistBins = 50000;

__global__ void k_asum_max_partial(const float2 *__restrict__ z, int64_t n, double *__restrict__ part) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = z[i];
        acc += (double)fabsf(v.x) + (double)fabsf(v.y);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// a_i = |scale * z_i| (rounded as written); block maxima of a.
__global__ void k_abs_scaled(const float2 *__restrict__ z, int64_t n, float scale, float *__restrict__ a,
                             float *__restrict__ bmax) {
    __shared__ float sh[256];
    float mx = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = z[i];
        const float re = __fmul_rn(v.x, scale), im = __fmul_rn(v.y, scale);
        const float m = __fsqrt_rn(__fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)));
        a[i] = m;
        mx = fmaxf(mx, m);
    }
    sh[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) bmax[blockIdx.x] = sh[0];
}

__global__ void k_histogram(const float *__restrict__ a, int64_t n, float mx, unsigned int *__restrict__ hist) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float f = floorf(__fmul_rn(__fdiv_rn(a[i], mx), (float)kHistBins));
        unsigned int b = f >= (float)kHistBins ? (unsigned int)(kHistBins - 1) : (unsigned int)f;
        atomicAdd(&hist[b], 1u);
    }
}

__global__ void k_reciprocal_offset(float *__restrict__ a, int64_t n, float offset) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = a[i];
        if (offset > 0.f) v = __fadd_rn(v, offset);
        a[i] = __fdiv_rn(1.f, v);
    }
}

__global__ void k_precond_weights(const float2 *__restrict__ csm, int nb, int64_t nn, const float *__restrict__ reg,
                                  float kappa, float *__restrict__ w) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < nb; c++) {
            const float2 v = csm[(int64_t)c * nn + i];
            s = __fadd_rn(s, __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)));
        }
        if (reg) s = __fadd_rn(s, __fmul_rn(reg[i], kappa));
        w[i] = __fdiv_rn(1.f, __fsqrt_rn(s));
    }
}

unsigned int blocks_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned int)(b < 1184 ? (b < 1 ? 1 : b) : 1184);
}

}  // namespace

float image_operator_compute(const float2 *reg, int64_t n, bool offset_estimation, float *image,
                             cudaStream_t st) {
    if (!reg || !image || n <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid image operator arguments");
    const unsigned int nbk = blocks_for(n);
    DevBuf<double> part;
    part.ensure(nbk);
    DevBuf<float> bmax;
    bmax.ensure(nbk);
    k_asum_max_partial<<<nbk, 256, 0, st>>>(reg, n, part.get()); note_launch();
    GB_CUDA(cudaGetLastError());
    std::vector<double> hp(nbk);
    GB_CUDA(cudaMemcpyAsync(hp.data(), part.get(), nbk * sizeof(double), cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    double asum = 0.0;
    for (double v : hp) asum += v;
    if (!(asum > 0.0)) fail(GB_ERR_INVALID_ARGUMENT, "regularisation image is zero");
    const float scale = (float)n / (float)asum;
    k_abs_scaled<<<nbk, 256, 0, st>>>(reg, n, scale, image, bmax.get()); note_launch();
    GB_CUDA(cudaGetLastError());
    float offset = 0.f;
    if (offset_estimation) {
        std::vector<float> hm(nbk);
        GB_CUDA(cudaMemcpyAsync(hm.data(), bmax.get(), nbk * sizeof(float), cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaStreamSynchronize(st));
        float mx = 0.f;
        for (float v : hm) mx = v > mx ? v : mx;
        if (!(mx > 0.f)) fail(GB_ERR_INVALID_ARGUMENT, "regularisation image is zero");
        DevBuf<unsigned int> hist;
        hist.ensure(kHistBins);
        GB_CUDA(cudaMemsetAsync(hist.get(), 0, kHistBins * sizeof(unsigned int), st));
        k_histogram<<<nbk, 256, 0, st>>>(image, n, mx, hist.get()); note_launch();
        GB_CUDA(cudaGetLastError());
        std::vector<unsigned int> hh(kHistBins);
        GB_CUDA(cudaMemcpyAsync(hh.data(), hist.get(), kHistBins * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaStreamSynchronize(st));
        const unsigned int target = (unsigned int)(0.01f * (float)n);
        unsigned int cumsum = 0, counter = 0;
        while (cumsum < target && counter < (unsigned int)kHistBins) cumsum += hh[counter++];
        offset = (float)(counter + 1) * mx / (float)kHistBins;
    }
    k_reciprocal_offset<<<nbk, 256, 0, st>>>(image, n, offset); note_launch();
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaStreamSynchronize(st));   // the scratch buffers are freed on return
    return offset;
}

void sense_precond_weights(const float2 *csm, int nb, int64_t nn, const float *reg, float kappa, float *w,
                           cudaStream_t st) {
    if (!csm || !w || nb <= 0 || nn <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid preconditioner arguments");
    k_precond_weights<<<blocks_for(nn), 256, 0, st>>>(csm, nb, nn, reg, kappa, w); note_launch();
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
