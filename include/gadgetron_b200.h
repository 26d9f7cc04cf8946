/*
 * gadgetron_b200 — C ABI of the B200 (sm_100a) non-Cartesian reconstruction
 * path: Kaiser-Bessel NUFFT (gridding NC2C, degridding C2NC, deapodization,
 * zero-pad/crop around the oversampled FFT), the non-Cartesian SENSE operator
 * and the CG-SENSE solver.
 *
 * Conventions
 *   - Every entry point returns gb_status (GB_OK == 0); no C++ exception
 *     crosses this boundary.  gb_last_error_message() describes the last
 *     failure on the calling thread.
 *   - All array arguments are DEVICE pointers owned by the caller, on the
 *     device that was current when the object was created.  Complex data is
 *     interleaved float pairs {re, im} (Gadgetron's complext<float>).
 *   - Layouts are those of the reference arrays, x fastest:
 *       image          [N_0, ..., N_{D-1}, frames, batches]
 *       oversampled    [mos_0, ..., mos_{D-1}, frames, batches]
 *       samples        [M_total, batches] where frame f owns samples
 *                      [frame_offsets[f], frame_offsets[f+1])  (for equal
 *                      frames this is the reference [M, frames, batches])
 *       trajectory     [M_total] of D floats in [-1/2, 1/2]
 *       dcw            [M_total] floats (broadcast over batches)
 *       csm            [N_0, ..., N_{D-1}, coils]
 *   - A stream argument of 0 means the legacy default stream (what the
 *     reference uses everywhere).
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the Gadgetron source tree).
 */
#ifndef GADGETRON_B200_H
#define GADGETRON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define GB_API __declspec(dllexport)
#else
#define GB_API __attribute__((visibility("default")))
#endif

typedef enum gb_status {
    GB_OK = 0,
    GB_ERR_INVALID_ARGUMENT = 1,  /* bad size, NULL pointer, unsupported D   */
    GB_ERR_TRAJECTORY_RANGE = 2,  /* trajectory outside [-1/2, 1/2]          */
    GB_ERR_NOT_PREPROCESSED = 3,  /* compute before preprocess               */
    GB_ERR_CUDA = 4,              /* CUDA runtime error                      */
    GB_ERR_CUFFT = 5,             /* cuFFT error                             */
    GB_ERR_OUT_OF_MEMORY = 6,     /* device allocation failed                */
    GB_ERR_DIMENSION_MISMATCH = 7,/* array sizes disagree with the plan      */
    GB_ERR_TIMEOUT = 8,           /* a bounded device wait gave up           */
    GB_ERR_INTERNAL = 9
} gb_status;

/* Mirrors NFFT_comp_mode (toolboxes/nfft/NFFT.h:29-34). */
typedef enum gb_comp_mode {
    GB_FORWARDS_C2NC = 0,
    GB_FORWARDS_NC2C = 1,
    GB_BACKWARDS_C2NC = 2,
    GB_BACKWARDS_NC2C = 3
} gb_comp_mode;

/* Mirrors NFFT_prep_mode (toolboxes/nfft/NFFT.h:39-43). */
typedef enum gb_prep_mode { GB_PREP_C2NC = 0, GB_PREP_NC2C = 1, GB_PREP_ALL = 2 } gb_prep_mode;

/* Mirrors NFFT_conv_mode (toolboxes/nfft/NFFT.h:20-23). */
typedef enum gb_conv_mode { GB_CONV_C2NC = 0, GB_CONV_NC2C = 1 } gb_conv_mode;

/* Mirrors NFFT_fft_mode (toolboxes/nfft/NFFT.h:14-17). */
typedef enum gb_fft_mode { GB_FFT_FORWARDS = 0, GB_FFT_BACKWARDS = 1 } gb_fft_mode;

/* Plan flags. */
#define GB_FLAG_COMPENSATED 0x1u   /* compensated (TwoSum) in-tile accumulation */
#define GB_FLAG_AUTOTUNE    0x2u   /* autotune at preprocess (plans: 1 batch; SENSE: its coils) */
/* 3D gridding (NC2C) folds the padding ring as the reference's wrap_image_kernel
 * does (toolboxes/nfft/gpu/ConvolverNC2C_standard.cuh:394-437) instead of
 * periodically: on cells within the ring width of a z face it adds some
 * periodic images twice and others not at all (its dimension test
 * `i & combination`, :411-413).  For callers that need the reference's 3D
 * adjoint bit for bit in the math (not in the rounding: the extra terms are
 * added with float atomics, so such results are not bitwise repeatable).
 * No effect in 1D and 2D, where the reference's fold is the periodic one. */
#define GB_FLAG_REFERENCE_FOLD 0x4u

typedef struct gb_nufft_plan_s *gb_nufft_plan;
typedef struct gb_sense_op_s *gb_sense_op;
typedef struct gb_cg_solver_s *gb_cg_solver;
typedef struct gb_sense_buffer_s *gb_sense_buffer;

GB_API const char *gb_last_error_message(void);
GB_API const char *gb_version(void);

/* Number of CUDA kernels of this library launched so far in the process
 * (kernels inside a replayed CUDA graph count once per replay; cuFFT's own
 * kernels are not counted).  Instrumentation, no reference counterpart. */
GB_API uint64_t gb_kernel_launch_count(void);

/* ------------------------------------------------------------------ NUFFT */

/* Replaces NFFT<cuNDArray,float,D>::make_plan(matrix_size, matrix_size_os, W,
 * ConvolutionType) (toolboxes/nfft/gpu/cuNFFT.h:113-121, cuNFFT.cu:206-218)
 * and the checks of cuGriddingConvolution::initialize
 * (toolboxes/nfft/gpu/cuGriddingConvolution.cu:56-125): W >= 1.8, sizes
 * multiples of 32, mos >= N.  D in {1, 2, 3}. */
GB_API gb_status gb_nufft_plan_create(int D, const uint64_t *matrix_size,
                                      const uint64_t *matrix_size_os, float W,
                                      uint32_t flags, gb_nufft_plan *plan);

/* Replaces the plan's destructor (cuNFFT.cu:53-56). */
GB_API gb_status gb_nufft_plan_destroy(gb_nufft_plan plan);

/* Replaces NFFT_plan::preprocess(trajectory, NFFT_prep_mode)
 * (toolboxes/nfft/NFFT.h:67-68, NFFT.hpp:41-63) and
 * cuGriddingConvolution::preprocess (cuGriddingConvolution.cu:128-188).
 * trajectory: device, M_total D-vectors.  frame_offsets: HOST array of
 * num_frames+1 sample offsets (frame f owns [off[f], off[f+1])); pass NULL
 * for num_frames equal frames of M_total/num_frames samples each (the
 * reference's only form).  Returns GB_ERR_TRAJECTORY_RANGE when a coordinate
 * lies outside [-1/2, 1/2] (the reference throws std::runtime_error). */
GB_API gb_status gb_nufft_preprocess(gb_nufft_plan plan, const float *trajectory,
                                     uint64_t num_samples_total, uint32_t num_frames,
                                     const uint64_t *frame_offsets, gb_prep_mode mode,
                                     void *stream);

/* Replaces NFFT_plan::compute(in, out, dcw, NFFT_comp_mode)
 * (toolboxes/nfft/NFFT.h:77-78, NFFT.hpp:105-203).  The image side is the
 * matrix size, or the oversampled size when image_oversampled != 0 (the
 * reference decides by comparing array dimensions, NFFT.hpp:110-111).
 * num_batches is the product of the dimensions beyond frames.  dcw may be
 * NULL.  GB_BACKWARDS_C2NC is rejected (its reference form passes swapped
 * arguments, NFFT.hpp:233-239). */
GB_API gb_status gb_nufft_compute(gb_nufft_plan plan, const void *in, void *out,
                                  const float *dcw, gb_comp_mode mode,
                                  uint32_t num_batches, int image_oversampled,
                                  void *stream);

/* Replaces NFFT_plan::mult_MH_M(in, out, dcw) (NFFT.h:88-90,
 * NFFT.hpp:90-102): FORWARDS_C2NC then BACKWARDS_NC2C, dcw applied in both,
 * with the intermediate samples kept in device workspace in tile order. */
GB_API gb_status gb_nufft_mult_MH_M(gb_nufft_plan plan, const void *in, void *out,
                                    const float *dcw, uint32_t num_batches,
                                    void *stream);

/* Replaces NFFT_plan::convolve(in, out, NFFT_conv_mode, accumulate)
 * (NFFT.h:103-105, GriddingConvolution.hpp:42-62): degridding (C2NC,
 * oversampled grid -> samples) or gridding (NC2C, samples -> oversampled
 * grid). */
GB_API gb_status gb_nufft_convolve(gb_nufft_plan plan, const void *in, void *out,
                                   gb_conv_mode mode, int accumulate,
                                   uint32_t num_batches, void *stream);

/* Gridding (NC2C convolution, samples -> oversampled grid) exactly as
 * gb_nufft_convolve with GB_CONV_NC2C, but without allocating device memory.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running in a host callback or a real-time thread with a fixed memory
 * budget, or under another allocator that must not be bypassed.  Its scratch (the partial tiles of heavily loaded tiles) is
 * a fixed 16 MiB array in device memory that each GPU loading this library
 * keeps until exit; a plan and batch count needing more is rejected with
 * GB_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress), so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller.  The plan must be preprocessed. */
GB_API gb_status gb_nufft_convolve_nc2c_noalloc(gb_nufft_plan plan, const void *samples,
                                                void *grid, int accumulate,
                                                uint32_t num_batches, void *stream);

/* Replaces cuNFFT_impl::fft(data, NFFT_fft_mode, do_scale)
 * (toolboxes/nfft/gpu/cuNFFT.cu:58-70 -> cuNDFFT::fft/ifft): centred C2C
 * transform over the D grid dimensions of an oversampled array, in place. */
GB_API gb_status gb_nufft_fft(gb_nufft_plan plan, void *data, gb_fft_mode mode,
                              int do_scale, uint32_t num_frames_x_batches,
                              void *stream);

/* Replaces cuNFFT_impl::deapodize(image, fourier_domain)
 * (toolboxes/nfft/gpu/cuNFFT.cu:74-92): in place, oversampled array. */
GB_API gb_status gb_nufft_deapodize(gb_nufft_plan plan, void *image, int fourier_domain,
                                    uint32_t num_frames_x_batches, void *stream);

/* Gradient of the forward NUFFT (FORWARDS_C2NC) with respect to the
 * trajectory.  For y = NUFFT_k(x) (dcw applied to the output when given),
 * writes grad_traj[j][d] = sum_b Re( w[b,j] * d y[b,j] / d k[j][d] ), i.e. the
 * real directional derivatives contracted with the caller's complex weights
 * w (for a real loss L and upstream gradient g = dL/d conj(y) x 2, pass
 * w = conj(g)).  image: [N..., frames, batches]; weights: samples layout;
 * grad_traj: [M_total][D] floats, overwritten.  No reference counterpart
 * (new surface for differentiation). */
GB_API gb_status gb_nufft_traj_grad(gb_nufft_plan plan, const void *image,
                                    const void *weights, const float *dcw,
                                    float *grad_traj, uint32_t num_batches,
                                    void *stream);

/* Same derivative, evaluated from an oversampled k-space grid that the caller
 * already holds (grid = FFT(deapodize(pad(x))), centred): grad_traj[j][d] =
 * sum_b Re( w[b,j] * sum_g d phi(s_j - g)/d k_d * grid[b,g] ).  Used for the
 * trajectory gradient of the adjoint.  No reference counterpart. */
GB_API gb_status gb_nufft_traj_grad_from_grid(gb_nufft_plan plan, const void *grid,
                                              const void *weights, float *grad_traj,
                                              uint32_t num_batches, void *stream);

/* Plan queries: get_matrix_size / get_matrix_size_os / get_W (NFFT.h:135-151),
 * plus the sample and frame counts recorded by preprocess. */
GB_API gb_status gb_nufft_get_info(gb_nufft_plan plan, int *D, uint64_t *matrix_size,
                                   uint64_t *matrix_size_os, float *W,
                                   uint64_t *num_samples_total, uint32_t *num_frames);

/* Device-side error word of the plan: kernels whose bounded waits ran out
 * (a bulk copy that did not complete, a grid barrier not reached by every
 * block) set a bit instead of spinning forever.  Synchronises the stream,
 * writes the word to *error_bits (0: none) and clears it.  No reference
 * counterpart. */
GB_API gb_status gb_nufft_device_errors(gb_nufft_plan plan, uint32_t *error_bits, void *stream);

/* Autotuner: on a preprocessed plan, times candidate tile shapes and coil
 * groups for num_batches batches (one gridding + one degridding pass each on
 * this trajectory) and keeps the fastest; the choice is cached per
 * (dimensions, sizes, W, frames, sample count, batches) for later plans.
 * Synchronises the stream.  No reference counterpart. */
GB_API gb_status gb_nufft_autotune(gb_nufft_plan plan, uint32_t num_batches, void *stream);

/* Diagnostic: device time (CUDA events on `stream`) of the two convolutions
 * inside the normal operator E^H E for `num_batches` batches -- degridding
 * into the plan's sample workspace with dcw applied twice (dcw may be NULL),
 * then gridding back into its k-space workspace -- launched `reps` times
 * each after one untimed round, exactly as E^H E launches them (same
 * kernels, same workspace layouts).  When flush is not NULL, flush_bytes of
 * it are overwritten before every launch so each one starts with a cold L2.
 * Averages in milliseconds; the workspaces' contents are overwritten.
 * Synchronises the stream.  No reference counterpart. */
GB_API gb_status gb_nufft_time_normal_convolutions(gb_nufft_plan plan, uint32_t num_batches, const float *dcw,
                                                   uint32_t reps, void *flush, uint64_t flush_bytes,
                                                   float *ms_grid, float *ms_degrid, void *stream);

/* Tile configuration used by the gridding kernels (chosen by the autotuner
 * when GB_FLAG_AUTOTUNE is set, else defaults), for inspection. */
GB_API gb_status gb_nufft_get_tiling(gb_nufft_plan plan, int *tile, int *coil_group);
GB_API gb_status gb_nufft_set_tiling(gb_nufft_plan plan, const int *tile, int coil_group);

/* How the normal operator (mult_MH_M, the CG-SENSE iteration) grids its own
 * tile-ordered samples: 0 (default) chooses by launch depth; 1 one CTA per
 * gridding work item; 2 one persistent launch whose CTAs take (frame, tile,
 * coil group) work units from a device-side queue.  Results are the same
 * bit for bit; only the speed differs.  Takes effect at the next launch (a
 * captured CG graph is re-captured).  No reference counterpart (tuning). */
GB_API gb_status gb_nufft_set_grid_schedule(gb_nufft_plan plan, int schedule);
GB_API gb_status gb_nufft_get_grid_schedule(gb_nufft_plan plan, int *schedule);

/* ------------------------------------------------------------------ SENSE */

/* Replaces cuNonCartesianSenseOperator<float,D>(ConvolutionType) + setup(
 * matrix_size, matrix_size_os, W) (toolboxes/mri/pmri/gpu/
 * cuNonCartesianSenseOperator.h:12-41, .cu:7-12,64-69). */
GB_API gb_status gb_sense_create(int D, const uint64_t *matrix_size,
                                 const uint64_t *matrix_size_os, float W,
                                 uint32_t flags, gb_sense_op *op);
GB_API gb_status gb_sense_destroy(gb_sense_op op);

/* Replaces cuNonCartesianSenseOperator::preprocess(trajectory) (.cu:71-84). */
GB_API gb_status gb_sense_preprocess(gb_sense_op op, const float *trajectory,
                                     uint64_t num_samples_total, uint32_t num_frames,
                                     const uint64_t *frame_offsets, void *stream);

/* Replaces senseOperator::set_csm (toolboxes/mri/pmri/gpu/senseOperator.h:26-35).
 * csm: [N..., num_coils] complex, device; the pointer is retained (not copied),
 * as the reference retains its shared_ptr. */
GB_API gb_status gb_sense_set_csm(gb_sense_op op, const void *csm, uint32_t num_coils);

/* Replaces cuNonCartesianSenseOperator::set_dcw (.cu:86-90).  dcw: [M_total]
 * floats, retained; NULL clears.  Callers pass sqrt(w) as the reference's
 * gadget does (gadgets/pmri/gpuCgSenseGadget.cpp:129). */
GB_API gb_status gb_sense_set_dcw(gb_sense_op op, const float *dcw);

/* Replaces mult_M(in, out, accumulate) (.cu:14-38): image [N..., frames] ->
 * samples [M_total, coils]. */
GB_API gb_status gb_sense_mult_M(gb_sense_op op, const void *in, void *out,
                                 int accumulate, void *stream);

/* Replaces mult_MH(in, out, accumulate) (.cu:40-62). */
GB_API gb_status gb_sense_mult_MH(gb_sense_op op, const void *in, void *out,
                                  int accumulate, void *stream);

/* Replaces linearOperator::mult_MH_M (toolboxes/operators/linearOperator.h:75-85)
 * for this operator, fused: the coil loop, FFTs and the sample round trip stay
 * in device workspace. */
GB_API gb_status gb_sense_mult_MH_M(gb_sense_op op, const void *in, void *out,
                                    int accumulate, void *stream);

GB_API gb_status gb_sense_get_nufft_plan(gb_sense_op op, gb_nufft_plan *plan);

/* Autotunes the operator's plan for its coil count (csm must be set). */
GB_API gb_status gb_sense_autotune(gb_sense_op op, void *stream);

/* --------------------------------------------------------------------- CG */

/* Replaces cuCgSolver<float_complext> (toolboxes/solvers/gpu/cuCgSolver.h:24-29)
 * with cgSolver's defaults (toolboxes/solvers/cgSolver.h:49-54): 10
 * iterations, tc_tolerance 1e-3, relative-residual stop rule. */
GB_API gb_status gb_cg_create(gb_cg_solver *solver);
GB_API gb_status gb_cg_destroy(gb_cg_solver solver);

/* set_encoding_operator (toolboxes/solvers/linearOperatorSolver.h:28-49).
 * weight mirrors generalOperator::set_weight (default 1). */
GB_API gb_status gb_cg_set_encoding_operator(gb_cg_solver solver, gb_sense_op op,
                                             float weight);
/* set_max_iterations / set_tc_tolerance (cgSolver.h:82-92). */
GB_API gb_status gb_cg_set_max_iterations(gb_cg_solver solver, uint32_t iterations);
GB_API gb_status gb_cg_set_tc_tolerance(gb_cg_solver solver, float tolerance);
/* set_x0 (toolboxes/solvers/solver.h:33-34); NULL clears.  Retained pointer. */
GB_API gb_status gb_cg_set_x0(gb_cg_solver solver, const void *x0);
/* cgPreconditioner::set_weights (toolboxes/solvers/cgPreconditioner.h:24-39):
 * real diagonal weights [N..., frames] (applied twice, as the reference does);
 * NULL clears.  Retained pointer. */
GB_API gb_status gb_cg_set_preconditioner(gb_cg_solver solver, const float *weights);
/* Kappa-weighted identity regulariser R = I: adds kappa * x to E^H E x
 * (cgSolver::add_regularization_operator with an identityOperator,
 * cgSolver.h:355-390).  0 disables. */
GB_API gb_status gb_cg_set_identity_regularization(gb_cg_solver solver, float kappa);
/* cgSolver::add_regularization_operator(R) with R a cuImageOperator of weight
 * kappa (gadgets/pmri/gpuCgSenseGadget.cpp:71-76; cgSolver.h:380-389;
 * imageOperator::mult_MH_M, imageOperator.h:48-67): adds
 * kappa * image^2 * x to E^H E x.  image: device floats [N..., frames] as made
 * by gb_image_operator_compute (retained pointer); kappa 0 disables. */
GB_API gb_status gb_cg_set_image_regularization(gb_cg_solver solver, const float *image, float kappa);
/* imageOperator::compute(reg_image, offset_estimation) with
 * cuImageOperator::estimate_offset (toolboxes/operators/imageOperator.h:27-45,
 * toolboxes/operators/gpu/cuImageOperator.h:35-62): image[i] =
 * 1 / (|reg[i] * n / asum(reg)| + offset), offset from the 1st percentile of
 * a 50000-bin histogram (0 without estimation).  reg: n complex64 (device);
 * image: n floats (device); offset: host float or NULL.  Synchronises. */
GB_API gb_status gb_image_operator_compute(const void *reg_image, uint64_t n, int offset_estimation,
                                           float *image, float *offset, void *stream);
/* ---------------------------------------------------- radial trajectories */

/* compute_radial_trajectory_golden_ratio_2d (toolboxes/core/gpu/radial_utilities.cu:46-87,
 * radial_utilities.h:16-39): trajectory [frames][profiles_per_frame *
 * samples_per_profile][2] floats (device), profile p (counted over all frames)
 * at angle (p + profile_offset) * step + pi, step = pi (3 - sqrt 5)/2 (mode 0,
 * GR_SMALLEST) or pi / golden ratio (mode 1, GR_ORIGINAL); sample s at
 * (s - S/2) / S.  samples_per_profile must be a multiple of 32. */
GB_API gb_status gb_radial_trajectory_golden_ratio_2d(uint32_t samples_per_profile, uint32_t profiles_per_frame,
                                                     uint32_t frames, uint32_t profile_offset, int mode,
                                                     float *trajectory, void *stream);
/* compute_radial_trajectory_fixed_angle_2d (radial_utilities.cu:143-199). */
GB_API gb_status gb_radial_trajectory_fixed_angle_2d(uint32_t samples_per_profile, uint32_t profiles_per_frame,
                                                     uint32_t frames, float angular_offset, float *trajectory,
                                                     void *stream);
/* compute_radial_trajectory_variable_angle_2d (radial_utilities.cu:89-140):
 * angles: device floats [frames]. */
GB_API gb_status gb_radial_trajectory_variable_angle_2d(const float *angles, uint32_t samples_per_profile,
                                                        uint32_t profiles_per_frame, uint32_t frames,
                                                        float *trajectory, void *stream);
/* compute_radial_dcw_golden_ratio_2d / compute_radial_dcw_fixed_angle_2d
 * (radial_utilities.cu:200-441): Voronoi-area weights of one frame,
 * dcw [profiles * samples_per_profile] floats (device). */
GB_API gb_status gb_radial_dcw_golden_ratio_2d(uint32_t samples_per_profile, uint32_t profiles, float alpha,
                                               float one_over_radial_oversampling, uint32_t profile_offset, int mode,
                                               float *dcw, void *stream);
GB_API gb_status gb_radial_dcw_fixed_angle_2d(uint32_t samples_per_profile, uint32_t profiles, float alpha,
                                              float one_over_radial_oversampling, float *dcw, void *stream);

/* ------------------------------------------------------ SENSE buffer --- */

/* cuSenseBuffer<float, D> (toolboxes/mri/pmri/gpu/cuSenseBuffer.h,
 * cuBuffer.h:13-57): a cycle of num_cycles + 1 oversampled k-space slots
 * [coils][mos...] filled by gridding (NC2C, accumulating) num_sub_cycles
 * frames each, and a running sum of the last num_cycles complete slots.
 * setup allocates and clears (cuBuffer::setup); the dcw and csm pointers are
 * retained.  add_frame_data: samples [coils][M] complex64, trajectory [M][D]
 * floats (device); *cycle_completed (may be NULL) = 1 when a slot completed
 * (cuBuffer::add_frame_data).  get_accumulated_coil_images: [coils][N...]
 * (centred backward FFT, deapodization, crop of the running sum; ones while
 * no slot has completed).  get_combined_coil_image: [N...] = sum_c
 * conj(csm_c) x the last accumulated coil images.  Normalisation factor
 * 1 / (num_cycles * num_sub_cycles) (cuBuffer::get_normalization_factor). */
GB_API gb_status gb_sense_buffer_create(gb_sense_buffer *buffer);
GB_API gb_status gb_sense_buffer_destroy(gb_sense_buffer buffer);
GB_API gb_status gb_sense_buffer_setup(gb_sense_buffer buffer, int D, const uint64_t *matrix_size,
                                       const uint64_t *matrix_size_os, float W, uint32_t num_coils,
                                       uint32_t num_cycles, uint32_t num_sub_cycles, void *stream);
GB_API gb_status gb_sense_buffer_clear(gb_sense_buffer buffer, void *stream);
GB_API gb_status gb_sense_buffer_set_dcw(gb_sense_buffer buffer, const float *dcw);
GB_API gb_status gb_sense_buffer_set_csm(gb_sense_buffer buffer, const void *csm);
GB_API gb_status gb_sense_buffer_add_frame_data(gb_sense_buffer buffer, const void *samples, const float *trajectory,
                                                uint64_t num_samples, int *cycle_completed, void *stream);
GB_API gb_status gb_sense_buffer_get_accumulated_coil_images(gb_sense_buffer buffer, void *images, void *stream);
GB_API gb_status gb_sense_buffer_get_combined_coil_image(gb_sense_buffer buffer, void *image, void *stream);
GB_API gb_status gb_sense_buffer_get_normalization_factor(gb_sense_buffer buffer, float *factor);

/* estimate_b1_map<float, D> (toolboxes/mri/pmri/gpu/b1_map.h:14-20,
 * b1_map.cu:29-118): coil sensitivities from coil images
 * [num_coils][image_size...] complex64 (device): RSS normalisation over the
 * first target_coils coils (all when target_coils <= 0 or larger), per-pixel
 * coil correlation matrices smoothed over a 7^D box (zero outside the
 * image), dominant eigenvector by two power iterations, phase of coil 0 set
 * to zero.  csm: [target][image_size...] complex64 (device); at most 32
 * target coils.  Synchronises. */
GB_API gb_status gb_estimate_b1_map(int D, const uint64_t *image_size, uint32_t num_coils, int target_coils,
                                    const void *coil_images, void *csm, void *stream);

/* estimate_dcw (toolboxes/mri/sdc/SDC.hpp:19-80, gpu/cuSDC.cu): iterative
 * density compensation with the Jinc kernel of width kernel_width (radius
 * 0.9696 * kernel_width) on a grid of round_up_32(N * os_factor) cells per
 * dimension: w <- w / C2NC(NC2C(w)), num_iterations times, from w = 1 or
 * initial_dcw (may be NULL).  trajectory: num_samples x D floats in
 * [-1/2, 1/2] (device); dcw: num_samples floats (device).  Synchronises. */
GB_API gb_status gb_sdc_estimate_dcw(int D, const uint64_t *matrix_size, float os_factor, uint32_t num_iterations,
                                     float kernel_width, const float *trajectory, uint64_t num_samples,
                                     const float *initial_dcw, float *dcw, void *stream);

/* Preconditioner weights of gpuCgSenseGadget.cpp:167-176:
 * w = 1 / sqrt(sum_c |csm_c|^2 + kappa * reg_image) over the N... pixels of
 * the operator (reg_image NULL: csm term only).  weights: device floats. */
GB_API gb_status gb_sense_precond_weights(gb_sense_op op, const float *reg_image, float kappa,
                                          float *weights, void *stream);
/* Outer iterative refinement: solve `refinements` times, each from the FP64
 * residual of the previous solution (x <- x + CG(E^H d - E^H E x)).  1 = off. */
GB_API gb_status gb_cg_set_refinements(gb_cg_solver solver, uint32_t refinements);
/* Diagnostic: how many times a block of the fused CG iteration polls the
 * grid barrier before it gives up (0 = the default, 2^26 polls, about 4 s).
 * A block that gives up sets bit 1 of the plan's device error word
 * (gb_nufft_device_errors) and carries on, so a solve never hangs; that
 * solve's values are void, and the next solve starts from cleared barrier
 * counters.  A small limit makes the timeout path run on purpose (tests).
 * No reference counterpart. */
GB_API gb_status gb_cg_set_barrier_spin_limit(gb_cg_solver solver, uint32_t spin_limit);

/* 2D plans under the project FFT passes run each CG iteration with the x
 * pass of the forward FFT fused into the direction update and pad, and the x
 * pass of the adjoint FFT fused into the crop, coil sum and <p,q> (plain
 * launches, no grid barrier): enable = 1, the default.  enable = 0 selects the
 * barrier-synchronised fused tail used by 3D plans instead.  Results agree to
 * rounding.  No reference counterpart (tuning, tests). */
GB_API gb_status gb_cg_set_row_fusion(gb_cg_solver solver, int enable);
/* Solve the frames of a multi-frame operator as independent problems: each
 * frame gets its own CG scalars (rq, alpha, beta, stop flag) while every
 * kernel still covers all frames in one launch.  0 (default) = the
 * reference's coupled solve over the whole multi-frame vector.  With 1, the
 * result equals one solve per frame.  No reference counterpart. */
GB_API gb_status gb_cg_set_frame_independent(gb_cg_solver solver, int independent);
/* Capture each CG iteration (all kernels and FFTs, no host synchronisation)
 * into one CUDA graph on first use and replay it; 0 = plain launches. */
GB_API gb_status gb_cg_set_use_graph(gb_cg_solver solver, int use_graph);

/* Replaces cgSolver::solve(d) (cgSolver.h:105-118): x = argmin ||E x - d||^2
 * by CG on E^H E x = E^H d.  d: samples [M_total, coils]; x_out: image
 * [N..., frames].  residual_history (device, optional, >= iterations*refinements
 * doubles) receives rq/rq0 per iteration.  Scalars stay on the device (FP64
 * dot products and norms); the call synchronises only at its end to report
 * the number of iterations run (iterations_run may be NULL). */
GB_API gb_status gb_cg_solve(gb_cg_solver solver, const void *d, void *x_out,
                             double *residual_history, uint32_t *iterations_run,
                             void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GADGETRON_B200_H */
