// extern "C" boundary: status codes instead of exceptions, thread-local
// error messages, caller-owned device pointers.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const std::string &msg) { g_last_error = msg; }

struct Failure {
    gb_status st;
    std::string msg;
};

void fail(gb_status st, const std::string &msg) { throw Failure{st, msg}; }

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GB_ERR_OUT_OF_MEMORY : GB_ERR_CUDA,
             std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void check_cufft(cufftResult r, const char *what) {
    if (r != CUFFT_SUCCESS)
        fail(r == CUFFT_ALLOC_FAILED ? GB_ERR_OUT_OF_MEMORY : GB_ERR_CUFFT,
             std::string(what) + ": cuFFT error " + std::to_string((int)r));
}

template <class F>
static gb_status guarded(F &&f) {
    try {
        f();
        return GB_OK;
    } catch (const Failure &e) {
        set_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return GB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception &e) {
        set_error(e.what());
        return GB_ERR_INTERNAL;
    } catch (...) {
        set_error("unknown error");
        return GB_ERR_INTERNAL;
    }
}

static cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Switches to the object's device for the duration of a call.
struct DeviceGuard {
    int old = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&old);
        if (old != dev) check_cuda(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceGuard() {
        int cur;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != old && old >= 0) cudaSetDevice(old);
    }
};

}  // namespace gb

using namespace gb;

struct gb_nufft_plan_s {
    std::unique_ptr<NufftPlan> owned;   // null for a view of an operator's plan
    NufftPlan *p = nullptr;
};
struct gb_sense_op_s {
    SenseOp s;
    gb_nufft_plan_s view;
};
struct gb_cg_solver_s {
    CgSolver c;
};
struct gb_sense_buffer_s {
    SenseBuffer b;
};

namespace gb {
NufftPlan *plan_from_handle(gb_nufft_plan h) { return h ? h->p : nullptr; }

// Maps the exception being handled to a status code and records its message
// (the same mapping the entry points of this file use).
gb_status current_exception_status() {
    try {
        throw;
    } catch (const Failure &e) {
        set_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return GB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception &e) {
        set_error(e.what());
        return GB_ERR_INTERNAL;
    } catch (...) {
        set_error("unknown error");
        return GB_ERR_INTERNAL;
    }
}
}  // namespace gb

extern "C" {

GB_API const char *gb_last_error_message(void) { return g_last_error.c_str(); }

GB_API const char *gb_version(void) { return "gadgetron_b200 0.1 (sm_100a)"; }

GB_API uint64_t gb_kernel_launch_count(void) { return launch_count(); }


GB_API gb_status gb_nufft_plan_create(int D, const uint64_t *matrix_size, const uint64_t *matrix_size_os,
                                      float W, uint32_t flags, gb_nufft_plan *plan) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan pointer");
        *plan = nullptr;
        auto *h = new gb_nufft_plan_s();
        h->owned.reset(new NufftPlan());
        h->p = h->owned.get();
        try {
            plan_init(*h->p, D, matrix_size, matrix_size_os, W, flags);
            plan_default_tiling(*h->p);
        } catch (...) {
            delete h;
            throw;
        }
        *plan = h;
    });
}

GB_API gb_status gb_nufft_plan_destroy(gb_nufft_plan plan) {
    return guarded([&] {
        if (!plan) return;
        if (!plan->owned) fail(GB_ERR_INVALID_ARGUMENT, "this plan belongs to a SENSE operator");
        DeviceGuard g((*plan->p).device);
        delete plan;
    });
}

GB_API gb_status gb_nufft_preprocess(gb_nufft_plan plan, const float *trajectory, uint64_t num_samples_total,
                                     uint32_t num_frames, const uint64_t *frame_offsets, gb_prep_mode mode,
                                     void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        plan_preprocess((*plan->p), trajectory, num_samples_total, num_frames, frame_offsets, mode, S(stream));
        if ((*plan->p).flags & GB_FLAG_AUTOTUNE) plan_autotune(*plan->p, 1, S(stream));
    });
}

GB_API gb_status gb_nufft_compute(gb_nufft_plan plan, const void *in, void *out, const float *dcw,
                                  gb_comp_mode mode, uint32_t num_batches, int image_oversampled, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        nufft_compute((*plan->p), in, out, dcw, mode, count_arg(num_batches, "number of batches"), image_oversampled != 0, S(stream));
    });
}

GB_API gb_status gb_nufft_mult_MH_M(gb_nufft_plan plan, const void *in, void *out, const float *dcw,
                                    uint32_t num_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        nufft_mult_MH_M((*plan->p), in, out, dcw, count_arg(num_batches, "number of batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_convolve(gb_nufft_plan plan, const void *in, void *out, gb_conv_mode mode,
                                   int accumulate, uint32_t num_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        nufft_convolve((*plan->p), in, out, mode, accumulate != 0, count_arg(num_batches, "number of batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_fft(gb_nufft_plan plan, void *data, gb_fft_mode mode, int do_scale,
                              uint32_t num_frames_x_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        nufft_fft((*plan->p), data, mode, do_scale != 0, count_arg(num_frames_x_batches, "number of frames x batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_deapodize(gb_nufft_plan plan, void *image, int fourier_domain,
                                    uint32_t num_frames_x_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        (void)fourier_domain;   // both filters carry the same real values
        DeviceGuard g((*plan->p).device);
        nufft_deapodize((*plan->p), image, count_arg(num_frames_x_batches, "number of frames x batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_traj_grad(gb_nufft_plan plan, const void *image, const void *weights, const float *dcw,
                                    float *grad_traj, uint32_t num_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        if (!image || !weights || !grad_traj) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        DeviceGuard g((*plan->p).device);
        nufft_traj_grad((*plan->p), static_cast<const float2 *>(image), static_cast<const float2 *>(weights), dcw,
                        grad_traj, count_arg(num_batches, "number of batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_traj_grad_from_grid(gb_nufft_plan plan, const void *grid, const void *weights,
                                              float *grad_traj, uint32_t num_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        if (!grid || !weights || !grad_traj) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        DeviceGuard g((*plan->p).device);
        nufft_traj_grad_from_grid((*plan->p), static_cast<const float2 *>(grid), static_cast<const float2 *>(weights),
                                  grad_traj, count_arg(num_batches, "number of batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_get_info(gb_nufft_plan plan, int *D, uint64_t *matrix_size, uint64_t *matrix_size_os,
                                   float *W, uint64_t *num_samples_total, uint32_t *num_frames) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        const NufftPlan &p = (*plan->p);
        if (D) *D = p.D;
        for (int d = 0; d < p.D; d++) {
            if (matrix_size) matrix_size[d] = (uint64_t)p.N[d];
            if (matrix_size_os) matrix_size_os[d] = (uint64_t)p.mos[d];
        }
        if (W) *W = p.W;
        if (num_samples_total) *num_samples_total = (uint64_t)p.Mtot;
        if (num_frames) *num_frames = p.F;
    });
}

GB_API gb_status gb_nufft_device_errors(gb_nufft_plan plan, uint32_t *error_bits, void *stream) {
    return guarded([&] {
        if (!plan || !error_bits) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        NufftPlan &p = *plan->p;
        DeviceGuard g(p.device);
        uint32_t bits = 0;
        if (p.err_flag.get()) {
            GB_CUDA(cudaMemcpyAsync(&bits, p.err_flag.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, S(stream)));
            GB_CUDA(cudaMemsetAsync(p.err_flag.get(), 0, sizeof(uint32_t), S(stream)));
            GB_CUDA(cudaStreamSynchronize(S(stream)));
        }
        *error_bits = bits;
    });
}

GB_API gb_status gb_nufft_autotune(gb_nufft_plan plan, uint32_t num_batches, void *stream) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        DeviceGuard g((*plan->p).device);
        plan_autotune(*plan->p, count_arg(num_batches, "number of batches"), S(stream));
    });
}

GB_API gb_status gb_nufft_time_normal_convolutions(gb_nufft_plan plan, uint32_t num_batches, const float *dcw,
                                                   uint32_t reps, void *flush, uint64_t flush_bytes,
                                                   float *ms_grid, float *ms_degrid, void *stream) {
    return guarded([&] {
        if (!plan || !ms_grid || !ms_degrid) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        DeviceGuard g((*plan->p).device);
        nufft_time_normal_convolutions(*plan->p, count_arg(num_batches, "number of batches"), dcw,
                                       count_arg(reps, "repetitions"), flush, (size_t)flush_bytes, ms_grid,
                                       ms_degrid, S(stream));
    });
}

GB_API gb_status gb_nufft_get_tiling(gb_nufft_plan plan, int *tile, int *coil_group) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        for (int d = 0; d < kMaxD; d++)
            if (tile) tile[d] = (*plan->p).tiling.tile[d];
        if (coil_group) *coil_group = (*plan->p).tiling.cg;
    });
}

GB_API gb_status gb_nufft_set_tiling(gb_nufft_plan plan, const int *tile, int coil_group) {
    return guarded([&] {
        if (!plan || !tile) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        DeviceGuard g((*plan->p).device);
        NufftPlan &p = (*plan->p);
        plan_set_tiling(p, tile, coil_group);
        if (p.prepped) {   // re-bin the stored trajectory with the new tiles
            std::vector<uint64_t> offs(p.frame_off.begin(), p.frame_off.end());
            plan_preprocess(p, p.traj_copy.get(), (uint64_t)p.Mtot, p.F, offs.data(), p.prep_mode, nullptr);
        }
    });
}

GB_API gb_status gb_nufft_set_grid_schedule(gb_nufft_plan plan, int schedule) {
    return guarded([&] {
        if (!plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        if (schedule < 0 || schedule > 2) fail(GB_ERR_INVALID_ARGUMENT, "schedule must be 0, 1 or 2");
        (*plan->p).tiling.schedule = schedule;
    });
}

GB_API gb_status gb_nufft_get_grid_schedule(gb_nufft_plan plan, int *schedule) {
    return guarded([&] {
        if (!plan || !schedule) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        *schedule = (*plan->p).tiling.schedule;
    });
}

// ---------------------------------------------------------------- SENSE ---

GB_API gb_status gb_sense_create(int D, const uint64_t *matrix_size, const uint64_t *matrix_size_os, float W,
                                 uint32_t flags, gb_sense_op *op) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator pointer");
        *op = nullptr;
        auto *h = new gb_sense_op_s();
        try {
            plan_init(h->s.plan, D, matrix_size, matrix_size_os, W, flags);
            plan_default_tiling(h->s.plan);
        } catch (...) {
            delete h;
            throw;
        }
        *op = h;
    });
}

GB_API gb_status gb_sense_destroy(gb_sense_op op) {
    return guarded([&] {
        if (!op) return;
        DeviceGuard g(op->s.plan.device);
        delete op;
    });
}

GB_API gb_status gb_sense_preprocess(gb_sense_op op, const float *trajectory, uint64_t num_samples_total,
                                     uint32_t num_frames, const uint64_t *frame_offsets, void *stream) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        if (!trajectory) fail(GB_ERR_INVALID_ARGUMENT, "cuNonCartesianSenseOperator: cannot preprocess 0x0 trajectory.");
        DeviceGuard g(op->s.plan.device);
        plan_preprocess(op->s.plan, trajectory, num_samples_total, num_frames, frame_offsets, GB_PREP_ALL,
                        S(stream));
        if ((op->s.plan.flags & GB_FLAG_AUTOTUNE) && op->s.csm && op->s.ncoils > 0)
            plan_autotune(op->s.plan, op->s.ncoils, S(stream));
    });
}

GB_API gb_status gb_sense_set_csm(gb_sense_op op, const void *csm, uint32_t num_coils) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        if (!csm || num_coils == 0)
            fail(GB_ERR_INVALID_ARGUMENT, "Error: senseOperator::set_csm : unexpected csm dimensionality");
        op->s.csm = static_cast<const float2 *>(csm);
        op->s.ncoils = (int)num_coils;
    });
}

GB_API gb_status gb_sense_set_dcw(gb_sense_op op, const float *dcw) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        op->s.dcw = dcw;
    });
}

GB_API gb_status gb_sense_mult_M(gb_sense_op op, const void *in, void *out, int accumulate, void *stream) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        DeviceGuard g(op->s.plan.device);
        sense_mult_M(op->s, in, out, accumulate != 0, S(stream));
    });
}

GB_API gb_status gb_sense_mult_MH(gb_sense_op op, const void *in, void *out, int accumulate, void *stream) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        DeviceGuard g(op->s.plan.device);
        sense_mult_MH(op->s, in, out, accumulate != 0, S(stream));
    });
}

GB_API gb_status gb_sense_mult_MH_M(gb_sense_op op, const void *in, void *out, int accumulate, void *stream) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        DeviceGuard g(op->s.plan.device);
        sense_mult_MH_M(op->s, in, out, accumulate != 0, S(stream));
    });
}

GB_API gb_status gb_sense_autotune(gb_sense_op op, void *stream) {
    return guarded([&] {
        if (!op) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator");
        if (!op->s.csm || op->s.ncoils <= 0) fail(GB_ERR_INVALID_ARGUMENT, "set_csm before autotune");
        DeviceGuard g(op->s.plan.device);
        plan_autotune(op->s.plan, op->s.ncoils, S(stream));
    });
}

GB_API gb_status gb_sense_get_nufft_plan(gb_sense_op op, gb_nufft_plan *plan) {
    return guarded([&] {
        if (!op || !plan) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        // A non-owning view of the operator's plan.
        op->view.p = &op->s.plan;
        *plan = &op->view;
    });
}

// ------------------------------------------------------------------- CG ---

GB_API gb_status gb_cg_create(gb_cg_solver *solver) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver pointer");
        *solver = new gb_cg_solver_s();
    });
}

GB_API gb_status gb_cg_destroy(gb_cg_solver solver) {
    return guarded([&] {
        if (!solver) return;
        if (solver->c.E) {
            DeviceGuard g(solver->c.E->plan.device);
            delete solver;
        } else {
            delete solver;
        }
    });
}

GB_API gb_status gb_cg_set_encoding_operator(gb_cg_solver solver, gb_sense_op op, float weight) {
    return guarded([&] {
        if (!solver || !op) fail(GB_ERR_INVALID_ARGUMENT, "NULL argument");
        solver->c.E = &op->s;
        solver->c.weight = weight;
    });
}

GB_API gb_status gb_cg_set_max_iterations(gb_cg_solver solver, uint32_t iterations) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.iterations = iterations;
    });
}

GB_API gb_status gb_cg_set_tc_tolerance(gb_cg_solver solver, float tolerance) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.tol = tolerance;
    });
}

GB_API gb_status gb_cg_set_x0(gb_cg_solver solver, const void *x0) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.x0 = static_cast<const float2 *>(x0);
    });
}

GB_API gb_status gb_cg_set_preconditioner(gb_cg_solver solver, const float *weights) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.precond = weights;
    });
}

GB_API gb_status gb_cg_set_identity_regularization(gb_cg_solver solver, float kappa) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.kappa = kappa;
        solver->c.reg = nullptr;
    });
}

GB_API gb_status gb_cg_set_image_regularization(gb_cg_solver solver, const float *image, float kappa) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        if (!image && kappa != 0.f) fail(GB_ERR_INVALID_ARGUMENT, "NULL regularisation image");
        solver->c.kappa = kappa;
        solver->c.reg = image;
    });
}

GB_API gb_status gb_radial_trajectory_golden_ratio_2d(uint32_t samples_per_profile, uint32_t profiles_per_frame,
                                                     uint32_t frames, uint32_t profile_offset, int mode,
                                                     float *trajectory, void *stream) {
    return guarded([&] {
        radial_traj_golden(trajectory, (int)samples_per_profile, (int)profiles_per_frame, (int)frames,
                           (int)profile_offset, mode, S(stream));
    });
}

GB_API gb_status gb_radial_trajectory_fixed_angle_2d(uint32_t samples_per_profile, uint32_t profiles_per_frame,
                                                     uint32_t frames, float angular_offset, float *trajectory,
                                                     void *stream) {
    return guarded([&] {
        radial_traj_fixed(trajectory, (int)samples_per_profile, (int)profiles_per_frame, (int)frames, angular_offset,
                          S(stream));
    });
}

GB_API gb_status gb_radial_trajectory_variable_angle_2d(const float *angles, uint32_t samples_per_profile,
                                                        uint32_t profiles_per_frame, uint32_t frames,
                                                        float *trajectory, void *stream) {
    return guarded([&] {
        radial_traj_variable(trajectory, angles, (int)samples_per_profile, (int)profiles_per_frame, (int)frames,
                             S(stream));
    });
}

GB_API gb_status gb_radial_dcw_golden_ratio_2d(uint32_t samples_per_profile, uint32_t profiles, float alpha,
                                               float one_over_radial_oversampling, uint32_t profile_offset, int mode,
                                               float *dcw, void *stream) {
    return guarded([&] {
        radial_dcw(dcw, (int)samples_per_profile, (int)profiles, alpha, one_over_radial_oversampling,
                   (int)profile_offset, true, mode, S(stream));
    });
}

GB_API gb_status gb_radial_dcw_fixed_angle_2d(uint32_t samples_per_profile, uint32_t profiles, float alpha,
                                              float one_over_radial_oversampling, float *dcw, void *stream) {
    return guarded([&] {
        radial_dcw(dcw, (int)samples_per_profile, (int)profiles, alpha, one_over_radial_oversampling, 0, false, 1,
                   S(stream));
    });
}

GB_API gb_status gb_sense_buffer_create(gb_sense_buffer *buffer) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer pointer");
        *buffer = new gb_sense_buffer_s();
    });
}

GB_API gb_status gb_sense_buffer_destroy(gb_sense_buffer buffer) {
    return guarded([&] { delete buffer; });
}

GB_API gb_status gb_sense_buffer_setup(gb_sense_buffer buffer, int D, const uint64_t *matrix_size,
                                       const uint64_t *matrix_size_os, float W, uint32_t num_coils,
                                       uint32_t num_cycles, uint32_t num_sub_cycles, void *stream) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer");
        buffer->b.setup(D, matrix_size, matrix_size_os, W, (int)num_coils, (int)num_cycles, (int)num_sub_cycles,
                        S(stream));
    });
}

GB_API gb_status gb_sense_buffer_clear(gb_sense_buffer buffer, void *stream) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer");
        if (!buffer->b.plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
        DeviceGuard g(buffer->b.plan->device);
        buffer->b.clear(S(stream));
    });
}

GB_API gb_status gb_sense_buffer_set_dcw(gb_sense_buffer buffer, const float *dcw) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer");
        buffer->b.dcw = dcw;
    });
}

GB_API gb_status gb_sense_buffer_set_csm(gb_sense_buffer buffer, const void *csm) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer");
        buffer->b.csm = static_cast<const float2 *>(csm);
    });
}

GB_API gb_status gb_sense_buffer_add_frame_data(gb_sense_buffer buffer, const void *samples, const float *trajectory,
                                                uint64_t num_samples, int *cycle_completed, void *stream) {
    return guarded([&] {
        if (!buffer) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer");
        if (!buffer->b.plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
        DeviceGuard g(buffer->b.plan->device);
        const bool c = buffer->b.add_frame_data(static_cast<const float2 *>(samples), trajectory,
                                                (int64_t)num_samples, S(stream));
        if (cycle_completed) *cycle_completed = c ? 1 : 0;
    });
}

GB_API gb_status gb_sense_buffer_get_accumulated_coil_images(gb_sense_buffer buffer, void *images, void *stream) {
    return guarded([&] {
        if (!buffer || !images) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer or images");
        if (!buffer->b.plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
        DeviceGuard g(buffer->b.plan->device);
        buffer->b.accumulated_coil_images(static_cast<float2 *>(images), S(stream));
    });
}

GB_API gb_status gb_sense_buffer_get_combined_coil_image(gb_sense_buffer buffer, void *image, void *stream) {
    return guarded([&] {
        if (!buffer || !image) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer or image");
        if (!buffer->b.plan) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
        DeviceGuard g(buffer->b.plan->device);
        buffer->b.combined_coil_image(static_cast<float2 *>(image), S(stream));
    });
}

GB_API gb_status gb_sense_buffer_get_normalization_factor(gb_sense_buffer buffer, float *factor) {
    return guarded([&] {
        if (!buffer || !factor) fail(GB_ERR_INVALID_ARGUMENT, "NULL buffer or factor");
        if (buffer->b.cycle_length < 2) fail(GB_ERR_INVALID_ARGUMENT, "cuBuffer: setup has not been called");
        *factor = 1.f / (((float)buffer->b.cycle_length - 1.f) * (float)buffer->b.sub_cycle_length);
    });
}

GB_API gb_status gb_estimate_b1_map(int D, const uint64_t *image_size, uint32_t num_coils, int target_coils,
                                    const void *coil_images, void *csm, void *stream) {
    return guarded([&] {
        estimate_b1_map(D, image_size, (int)num_coils, target_coils, static_cast<const float2 *>(coil_images),
                        static_cast<float2 *>(csm), S(stream));
    });
}

GB_API gb_status gb_sdc_estimate_dcw(int D, const uint64_t *matrix_size, float os_factor, uint32_t num_iterations,
                                     float kernel_width, const float *trajectory, uint64_t num_samples,
                                     const float *initial_dcw, float *dcw, void *stream) {
    return guarded([&] {
        sdc_estimate_dcw(D, matrix_size, os_factor, (int)num_iterations, kernel_width, trajectory,
                         (int64_t)num_samples, initial_dcw, dcw, S(stream));
    });
}

GB_API gb_status gb_image_operator_compute(const void *reg_image, uint64_t n, int offset_estimation,
                                           float *image, float *offset, void *stream) {
    return guarded([&] {
        if (!reg_image || !image || n == 0) fail(GB_ERR_INVALID_ARGUMENT, "invalid image operator arguments");
        const float off = image_operator_compute(static_cast<const float2 *>(reg_image), (int64_t)n,
                                                 offset_estimation != 0, image, S(stream));
        if (offset) *offset = off;
    });
}

GB_API gb_status gb_sense_precond_weights(gb_sense_op op, const float *reg_image, float kappa, float *weights,
                                          void *stream) {
    return guarded([&] {
        if (!op || !weights) fail(GB_ERR_INVALID_ARGUMENT, "NULL operator or weights");
        if (!op->s.csm || op->s.ncoils <= 0) fail(GB_ERR_INVALID_ARGUMENT, "set_csm before the preconditioner");
        sense_precond_weights(op->s.csm, op->s.ncoils, op->s.plan.kp.NN, reg_image, kappa, weights, S(stream));
    });
}

GB_API gb_status gb_cg_set_refinements(gb_cg_solver solver, uint32_t refinements) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        if (refinements == 0) fail(GB_ERR_INVALID_ARGUMENT, "refinements must be >= 1");
        solver->c.refinements = refinements;
    });
}

GB_API gb_status gb_cg_set_barrier_spin_limit(gb_cg_solver solver, uint32_t spin_limit) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.barrier_spin_limit = spin_limit;
    });
}

GB_API gb_status gb_cg_set_row_fusion(gb_cg_solver solver, int enable) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.row_fusion = enable != 0;
    });
}

GB_API gb_status gb_cg_set_frame_independent(gb_cg_solver solver, int independent) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.independent_frames = independent != 0;
    });
}

GB_API gb_status gb_cg_set_use_graph(gb_cg_solver solver, int use_graph) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        solver->c.use_graph = use_graph != 0;
    });
}

GB_API gb_status gb_cg_solve(gb_cg_solver solver, const void *d, void *x_out, double *residual_history,
                             uint32_t *iterations_run, void *stream) {
    return guarded([&] {
        if (!solver) fail(GB_ERR_INVALID_ARGUMENT, "NULL solver");
        if (!solver->c.E) fail(GB_ERR_INVALID_ARGUMENT, "Error: cgSolver::compute_rhs : no encoding operator is set");
        DeviceGuard g(solver->c.E->plan.device);
        cg_solve(solver->c, d, x_out, residual_history, iterations_run, S(stream));
    });
}

}  // extern "C"
