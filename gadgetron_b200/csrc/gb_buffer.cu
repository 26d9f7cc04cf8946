// Cyclic k-space accumulation buffer of the real-time SENSE pipelines
// (cuBuffer / cuSenseBuffer, toolboxes/mri/pmri/gpu/cuBuffer.cpp:7-195 and
// cuSenseBuffer.cpp:5-40): every frame's samples are gridded (NC2C,
// accumulating) into the current slot of a cycle of num_cycles + 1 oversampled
// k-space buffers; after num_sub_cycles frames the slot is added to a running
// sum and the next slot is subtracted from it and cleared, so the sum always
// holds the last num_cycles complete slots.  The accumulated coil images are
// the running sum transformed back (centred backward FFT, deapodization, crop);
// the combined image is their conjugate-coil-sensitivity sum.
#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

namespace {

__global__ void k_scale_samples(const float2 *__restrict__ in, const float *__restrict__ dcw, int nb, int64_t M,
                                float2 *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)nb * M) return;
    const float w = dcw[i % M];
    const float2 v = in[i];
    out[i] = make_float2(v.x * w, v.y * w);
}

// acc += cur; acc -= next
__global__ void k_cycle_update(float2 *__restrict__ acc, const float2 *__restrict__ cur,
                               const float2 *__restrict__ next, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 a = acc[i];
    const float2 c = cur[i];
    a.x += c.x;
    a.y += c.y;
    const float2 x = next[i];
    a.x -= x.x;
    a.y -= x.y;
    acc[i] = a;
}

__global__ void k_fill_c(float2 *p, int64_t n, float2 v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Centred crop [nb][mos...] -> [nb][N...] (offset (mos - N) / 2 per dimension).
__global__ void k_crop_std(KParams k, const float2 *__restrict__ in, int nb, float2 *__restrict__ out) {
    const int64_t n = (int64_t)nb * k.NN;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t b = i / k.NN;
    int64_t r = i - b * k.NN;
    const int x = (int)(r % k.N[0]);
    r /= k.N[0];
    const int y = (int)(r % k.N[1]);
    const int z = (int)(r / k.N[1]);
    const int gx = x + ((k.mos[0] - k.N[0]) >> 1), gy = y + ((k.mos[1] - k.N[1]) >> 1),
              gz = z + ((k.mos[2] - k.N[2]) >> 1);
    out[i] = in[b * k.G + ((int64_t)gz * k.mos[1] + gy) * k.mos[0] + gx];
}

// out = sum_c conj(csm_c) * img_c   (mult_csm_conj_sum, sense_utilities.cu:66-78)
__global__ void k_csm_conj_sum(const float2 *__restrict__ img, const float2 *__restrict__ csm, int nb, int64_t nn,
                               float2 *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    float2 s = make_float2(0.f, 0.f);
    for (int c = 0; c < nb; c++) {
        const float2 v = img[(int64_t)c * nn + i], m = csm[(int64_t)c * nn + i];
        s.x += m.x * v.x + m.y * v.y;
        s.y += m.x * v.y - m.y * v.x;
    }
    out[i] = s;
}

unsigned int blocks_of(int64_t n) { return (unsigned int)((n + 255) / 256); }

}  // namespace

void SenseBuffer::setup(int D_, const uint64_t *N, const uint64_t *mos, float W, int ncoils, int num_cycles,
                        int num_sub_cycles, cudaStream_t st) {
    if (ncoils <= 0 || num_cycles <= 0 || num_sub_cycles <= 0)
        fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer::setup: coils, cycles and sub-cycles must be positive");
    plan.reset(new NufftPlan());
    plan_init(*plan, D_, N, mos, W, 0);
    plan_default_tiling(*plan);
    D = D_;
    coils = ncoils;
    cycle_length = num_cycles + 1;   // one working buffer beside the num_cycles full ones
    sub_cycle_length = num_sub_cycles;
    const int64_t slot = (int64_t)coils * plan->kp.G;
    acc.ensure((size_t)slot);
    cyc.ensure((size_t)slot * cycle_length);
    has_acc_image = false;
    clear(st);
}

void SenseBuffer::clear(cudaStream_t st) {
    if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
    const int64_t slot = (int64_t)coils * plan->kp.G;
    GB_CUDA(cudaMemsetAsync(acc.get(), 0, (size_t)slot * sizeof(float2), st));
    GB_CUDA(cudaMemsetAsync(cyc.get(), 0, (size_t)slot * cycle_length * sizeof(float2), st));
    cur_idx = cur_sub_idx = 0;
    acc_empty = true;
}

bool SenseBuffer::add_frame_data(const float2 *samples, const float *traj, int64_t M, cudaStream_t st) {
    if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
    if (!samples || !traj || M <= 0) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer::add_frame_data: illegal input pointer");
    NufftPlan &p = *plan;
    const int64_t slot = (int64_t)coils * p.kp.G;
    float2 *cur = cyc.get() + (int64_t)cur_idx * slot;
    plan_preprocess(p, traj, (uint64_t)M, 1, nullptr, GB_PREP_NC2C, st);
    const float2 *in = samples;
    if (dcw) {
        scaled.ensure((size_t)coils * M);
        k_scale_samples<<<blocks_of((int64_t)coils * M), 256, 0, st>>>(samples, dcw, coils, M, scaled.get());
        note_launch();
        GB_CUDA(cudaGetLastError());
        in = scaled.get();
    }
    nufft_convolve(p, in, cur, GB_CONV_NC2C, true, coils, st);
    bool completed = false;
    if (cur_sub_idx == sub_cycle_length - 1) {
        completed = true;
        const int next_idx = (cur_idx + 1) % cycle_length;
        float2 *next = cyc.get() + (int64_t)next_idx * slot;
        k_cycle_update<<<blocks_of(slot), 256, 0, st>>>(acc.get(), cur, next, slot);
        note_launch();
        GB_CUDA(cudaGetLastError());
        GB_CUDA(cudaMemsetAsync(next, 0, (size_t)slot * sizeof(float2), st));
        acc_empty = false;
        cur_idx = next_idx;
    }
    cur_sub_idx = (cur_sub_idx + 1) % sub_cycle_length;
    return completed;
}

// Computes the accumulated coil images into the buffer's own image (kept for
// the combined image, as the reference keeps acc_image_) and copies them to
// `out` when given.
void SenseBuffer::accumulated_coil_images(float2 *out, cudaStream_t st) {
    if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
    NufftPlan &p = *plan;
    const int64_t nimg = (int64_t)coils * p.kp.NN;
    acc_image.ensure((size_t)nimg);
    if (acc_empty) {   // not ready: an image of ones, as the reference returns
        k_fill_c<<<blocks_of(nimg), 256, 0, st>>>(acc_image.get(), nimg, make_float2(1.f, 0.f));
        note_launch();
        GB_CUDA(cudaGetLastError());
    } else {
        const int64_t slot = (int64_t)coils * p.kp.G;
        work.ensure((size_t)slot);
        GB_CUDA(cudaMemcpyAsync(work.get(), acc.get(), (size_t)slot * sizeof(float2), cudaMemcpyDeviceToDevice, st));
        nufft_fft(p, work.get(), GB_FFT_BACKWARDS, true, coils, st);
        nufft_deapodize(p, work.get(), coils, st);
        k_crop_std<<<blocks_of(nimg), 256, 0, st>>>(p.kp, work.get(), coils, acc_image.get());
        note_launch();
        GB_CUDA(cudaGetLastError());
    }
    has_acc_image = true;
    if (out && out != acc_image.get())
        GB_CUDA(cudaMemcpyAsync(out, acc_image.get(), (size_t)nimg * sizeof(float2), cudaMemcpyDeviceToDevice, st));
}

// The conjugate-csm coil sum of the last accumulated coil images (computed
// now if there are none yet; cuSenseBuffer.cpp:18-35).
void SenseBuffer::combined_coil_image(float2 *out, cudaStream_t st) {
    if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
    if (!csm) fail(GB_ERR_INVALID_ARGUMENT, "cuSenseBuffer::get_combined_coil_image: csm not set");
    if (!has_acc_image) accumulated_coil_images(nullptr, st);
    NufftPlan &p = *plan;
    k_csm_conj_sum<<<blocks_of(p.kp.NN), 256, 0, st>>>(acc_image.get(), csm, coils, p.kp.NN, out);
    note_launch();
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
