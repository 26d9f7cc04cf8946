// Radial trajectories and their density compensation weights, generated on
// the device (the inputs a radial reconstruction feeds to preprocess and
// set_dcw).  Behaviour of toolboxes/core/gpu/radial_utilities.cu:
//
//   golden ratio:   profile p (counted over all frames), sample s of S:
//                   angle = (p + profile_offset) * step + pi,
//                   k = (s - S/2) * (cos, sin)(angle) / S,
//                   step = pi (3 - sqrt 5) / 2 (smallest) or pi / ((sqrt 5 + 1) / 2) (original)
//                   (radial_utilities.cu:25-44);
//   fixed angle:    profile l of P in frame f of F:
//                   angle = (l + f / F) / P * pi + angular_offset + pi (:143-163);
//   variable angle: every profile of frame f at angle angles[f] (:89-105);
//   dcw:            the area of the "Voronoi polygon" of each sample: the
//                   midpoints towards its two neighbours on the profile and
//                   the nearest sample (with both neighbours along that
//                   profile) on either side of it, over all other profiles
//                   and both of their half-lines; the centre sample gets
//                   pi r^2 / P with r = alpha / (2 * radial oversampling)
//                   (:200-396).  Profile angles here have no + pi.
//
// Float arithmetic in the same order; a*b+c is one fused multiply-add, as
// nvcc contracts it by default.
#include <cfloat>

#include "gb_internal.cuh"

namespace gb {

namespace {

constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ float gr_step(int mode) {
    return mode == 0 ? kPiF * (3.0f - sqrtf(5.0f)) * 0.5f : kPiF / ((sqrtf(5.0f) + 1.0f) * 0.5f);
}

__device__ __forceinline__ void store_pos(float *traj, int64_t idx, float s, float bias, float S, float c, float sn) {
    traj[2 * idx] = (s - bias) * c / S;
    traj[2 * idx + 1] = (s - bias) * sn / S;
}

// one thread per sample; total = S * profiles_total
__global__ void k_traj_golden(float *traj, int S, int64_t total, float offset, int mode) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int64_t prof = idx / S;
    const float s = (float)(idx - prof * S);
    const float Sf = (float)S, bias = Sf * 0.5f;
    float sn, c;
    sincosf(fmaf((float)prof + offset, gr_step(mode), kPiF), &sn, &c);
    store_pos(traj, idx, s, bias, Sf, c, sn);
}

__global__ void k_traj_fixed(float *traj, int S, int P, int F, float angular_offset) {
    const int64_t total = (int64_t)S * P * F;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int64_t prof_all = idx / S;
    const float s = (float)(idx - prof_all * S);
    const int frame = (int)(prof_all / P), l = (int)(prof_all - (int64_t)frame * P);
    const float Sf = (float)S, bias = Sf * 0.5f;
    const float inv_p = 1.0f / (float)P, inv_f = 1.0f / (float)F;
    const float a = fmaf((float)frame, inv_f, (float)l) * inv_p;
    float sn, c;
    sincosf(fmaf(a, kPiF, angular_offset) + kPiF, &sn, &c);
    store_pos(traj, idx, s, bias, Sf, c, sn);
}

__global__ void k_traj_variable(float *traj, const float *angles, int S, int P, int F) {
    const int64_t total = (int64_t)S * P * F;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int64_t prof_all = idx / S;
    const float s = (float)(idx - prof_all * S);
    const int frame = (int)(prof_all / P);
    const float Sf = (float)S, bias = Sf * 0.5f;
    const float ang = angles[frame];
    store_pos(traj, idx, s, bias, Sf, cosf(ang), sinf(ang));
}

struct P2 {
    float x, y;
};
__device__ __forceinline__ float nsq(P2 a, P2 b) {
    const float dx = a.x - b.x, dy = a.y - b.y;
    return fmaf(dx, dx, dy * dy);
}

// One thread per sample.  Profile directions are computed once per CTA into
// shared memory (the same sincosf calls every thread would make).
__global__ void k_radial_dcw(float *dcw, int S, int P, float alpha, float ovs, float offset, int golden, int mode) {
    extern __shared__ float2 dirs[];   // [P] (cos, sin)
    const float step = golden ? gr_step(mode) : 0.f;
    const float inv_p = 1.0f / (float)P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        float sn, c;
        if (golden) sincosf(((float)i + offset) * step, &sn, &c);
        else sincosf((float)i * inv_p * kPiF, &sn, &c);
        dirs[i] = make_float2(c, sn);
    }
    __syncthreads();
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)S * P) return;
    const int prof = (int)(idx / S), si = (int)(idx - (int64_t)prof * S);
    const float Sf = (float)S, bias = Sf * 0.5f, s = (float)si;
    float w;
    if (si == S / 2) {
        const float r = (alpha * ovs) * 0.5f;
        w = r * r * kPiF / (float)P;
    } else {
        const float ctr = alpha * ((s - bias) * ovs);
        const float ctr_inv = alpha * ((Sf - s - bias) * ovs);
        const float prv = alpha * ((s - bias - 1.f) * ovs);
        const float prv_inv = alpha * ((Sf - (s - 1.f) - bias) * ovs);
        const float nxt = alpha * ((s - bias + 1.f) * ovs);
        const float nxt_inv = alpha * ((Sf - (s + 1.f) - bias) * ovs);
        const float2 d0 = dirs[prof];
        const P2 pos{ctr * d0.x, ctr * d0.y};
        const P2 nrm{-d0.y, d0.x};
        const P2 prev_own{prv * d0.x, prv * d0.y}, next_own{nxt * d0.x, nxt * d0.y};
        // nearest profile sample on each side: (previous, centre, next)
        P2 a0{FLT_MAX, FLT_MAX}, a1{FLT_MAX, FLT_MAX}, a2{FLT_MAX, FLT_MAX};
        P2 b0{FLT_MAX, FLT_MAX}, b1{FLT_MAX, FLT_MAX}, b2{FLT_MAX, FLT_MAX};
        for (int i = 0; i < P; i++) {
            if (i == prof) continue;
            const float2 d = dirs[i];
            for (int half = 0; half < 2; half++) {
                const float cs = half ? ctr_inv : ctr, ps = half ? prv_inv : prv, ns = half ? nxt_inv : nxt;
                const P2 cpos{cs * d.x, cs * d.y};
                const float side = fmaf(cpos.x - pos.x, nrm.x, (cpos.y - pos.y) * nrm.y);
                const float dist = nsq(cpos, pos);
                if (side > 0.f) {
                    if (dist < nsq(a1, pos)) {
                        a0 = P2{ps * d.x, ps * d.y};
                        a1 = cpos;
                        a2 = P2{ns * d.x, ns * d.y};
                    }
                } else if (dist < nsq(b1, pos)) {
                    b0 = P2{ps * d.x, ps * d.y};
                    b1 = cpos;
                    b2 = P2{ns * d.x, ns * d.y};
                }
            }
        }
        // polygon around the sample: own previous, side-a previous, centre,
        // next, own next, side-b next, centre, previous
        const P2 v[8] = {prev_own, a0, a1, a2, next_own, b2, b1, b0};
        float area = 0.f;
        P2 m[8];
        for (int k = 0; k < 8; k++) m[k] = P2{0.5f * (pos.x + v[k].x), 0.5f * (pos.y + v[k].y)};
        for (int k = 0; k < 8; k++) {
            const P2 u = m[k], t = m[(k + 1) & 7];
            area += u.x * t.y - t.x * u.y;
        }
        w = 0.5f * area;
        if (w < 0.f) w = -w;
    }
    dcw[idx] = w;
}

unsigned int blocks(int64_t n, int t) { return (unsigned int)((n + t - 1) / t); }

}  // namespace

void radial_traj_golden(float *traj, int S, int P, int F, int profile_offset, int mode, cudaStream_t st) {
    if (!traj || S <= 0 || P <= 0 || F <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid trajectory arguments");
    if (mode != 0 && mode != 1) fail(GB_ERR_INVALID_ARGUMENT, "golden ratio mode must be 0 (smallest) or 1 (original)");
    if (S % 32)
        fail(GB_ERR_INVALID_ARGUMENT, "compute_radial_trajectory_golden_ratio_2d: #samples/profile is not a multiple of the device's warp size.");
    const int64_t total = (int64_t)S * P * F;
    k_traj_golden<<<blocks(total, 256), 256, 0, st>>>(traj, S, total, (float)profile_offset, mode); note_launch();
    GB_CUDA(cudaGetLastError());
}

void radial_traj_fixed(float *traj, int S, int P, int F, float angular_offset, cudaStream_t st) {
    if (!traj || S <= 0 || P <= 0 || F <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid trajectory arguments");
    if (S % 32)
        fail(GB_ERR_INVALID_ARGUMENT, "Error:: compute_radial_trajectory_fixed_angle_2d: #samples/profile is not a multiple of the device's warp size.");
    k_traj_fixed<<<blocks((int64_t)S * P * F, 256), 256, 0, st>>>(traj, S, P, F, angular_offset); note_launch();
    GB_CUDA(cudaGetLastError());
}

void radial_traj_variable(float *traj, const float *angles, int S, int P, int F, cudaStream_t st) {
    if (!traj || !angles || S <= 0 || P <= 0 || F <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid trajectory arguments");
    if (S % 32)
        fail(GB_ERR_INVALID_ARGUMENT, "Error:: compute_radial_trajectory_fixed_angle_2d: #samples/profile is not a multiple of the device's warp size.");
    k_traj_variable<<<blocks((int64_t)S * P * F, 256), 256, 0, st>>>(traj, angles, S, P, F); note_launch();
    GB_CUDA(cudaGetLastError());
}

void radial_dcw(float *dcw, int S, int P, float alpha, float ovs, int profile_offset, bool golden, int mode,
                cudaStream_t st) {
    if (!dcw || S <= 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid dcw arguments");
    if (P < 4) fail(GB_ERR_INVALID_ARGUMENT, "Error:: compute_radial_dcw_<*>_2d: use at least four profiles");
    if (S % 2) fail(GB_ERR_INVALID_ARGUMENT, "Error:: compute_radial_dcw_<*>_2d: samples/profile must be even.");
    if (S % 32)
        fail(GB_ERR_INVALID_ARGUMENT, "Error:: compute_radial_dcw_<*>_2d: samples/profile number a multiple of the device's warp size.");
    if (golden && mode != 0 && mode != 1)
        fail(GB_ERR_INVALID_ARGUMENT, "compute_radial_dcw_golden_ratio_2d() :: unexpected mode");
    const size_t smem = (size_t)P * sizeof(float2);
    if (smem > 200 * 1024) fail(GB_ERR_INVALID_ARGUMENT, "too many profiles for the dcw kernel");
    if (smem > 48 * 1024) GB_CUDA(cudaFuncSetAttribute(k_radial_dcw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_radial_dcw<<<blocks((int64_t)S * P, 256), 256, smem, st>>>(dcw, S, P, alpha, ovs, (float)profile_offset,
                                                               golden ? 1 : 0, mode); note_launch();
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
