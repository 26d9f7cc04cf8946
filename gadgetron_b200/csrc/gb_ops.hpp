// Host-side objects behind the C ABI: the SENSE operator and the CG solver,
// plus the NUFFT operation entry points used by the ABI layer.
#pragma once

#include <memory>

#include "gb_internal.cuh"

namespace gb {

struct SenseOp {
    NufftPlan plan;
    const float2 *csm = nullptr;
    int ncoils = 0;
    const float *dcw = nullptr;
};

struct GraphKey {
    const void *d, *x;
    const double *hist;
    uint32_t iterations, refinements;
    const float2 *x0;
    const float *precond;
    const float *reg;
    float kappa, weight, tol;
    const float2 *csm;
    const float *dcw;
    int ncoils;
    uint64_t generation;
    bool independent;
    uint32_t spin_limit;
    bool row_fusion;
    bool operator==(const GraphKey &o) const {
        return generation == o.generation && independent == o.independent && spin_limit == o.spin_limit &&
               row_fusion == o.row_fusion && d == o.d && x == o.x && hist == o.hist && iterations == o.iterations &&
               refinements == o.refinements && x0 == o.x0 && precond == o.precond && reg == o.reg && kappa == o.kappa &&
               weight == o.weight && tol == o.tol && csm == o.csm && dcw == o.dcw && ncoils == o.ncoils;
    }
};

struct CgSeg;
struct CgGlobal;

struct CgSolver {
    SenseOp *E = nullptr;
    float weight = 1.f;
    uint32_t iterations = 10;      // cgSolver.h:51
    float tol = 1e-3f;             // cgSolver.h:52
    const float2 *x0 = nullptr;
    const float *precond = nullptr;
    float kappa = 0.f;
    // Image regulariser R = diag(reg) ([frames][N], null: R = I): the
    // operator gets kappa * R^H R = kappa * reg^2 (imageOperator::mult_MH_M).
    const float *reg = nullptr;
    uint32_t refinements = 1;
    bool use_graph = false;
    bool independent_frames = false;   // per-frame CG scalars (frames solved independently)
    // Polls of the fused tail's grid barrier before a block gives up (0: the
    // default of 2^26, about 4 s); a diagnostic setting, see
    // gb_cg_set_barrier_spin_limit.
    uint32_t barrier_spin_limit = 0;
    int nseg = 1;
    int64_t seg_len = 0;

    DevBuf<float2> x, r, p, q, rhs0, rhs;
    DevBuf<double2> x64, partials, partials2;
    DevBuf<unsigned int> tail_bar;   // grid barrier of the fused iteration tail
    int tail_tpp = 1;                // threads per pixel of the tail's coil sums
    bool use_rows = false;           // 2D: iteration with the row passes fused (no grid barrier)
    bool row_fusion = true;          // allow it (tests compare against the cooperative tail)
    bool rows_fold = false;          // with it: the x, r, p update folded into the next pad
    bool use_tail = false;           // fused tail (cooperative launch) available for this shape
    dim3 tail_grid;                  // its launch grid (blocks per segment, segments)
    DevBuf<CgSeg> segs;
    DevBuf<CgGlobal> G;
    cudaGraphExec_t graph_exec = nullptr;
    GraphKey graph_key{};
    uint64_t graph_kernels = 0;   // kernels of this library inside the graph
    ~CgSolver();
};

// NUFFT operations
float2 *ensure_img_os(NufftPlan &p, int64_t nbf, cudaStream_t st);
float2 *ensure_kgrid(NufftPlan &p, int64_t nbf);
float2 *ensure_samp(NufftPlan &p, int nb);
void launch_grid_prepare(NufftPlan &p, int nb, cudaStream_t st);
void nufft_forward(NufftPlan &p, const float2 *img, const float2 *csm, int nb, bool img_os, float2 *samples,
                   SampleLayout layout, const float *dcw, int dcw_pow, bool accumulate, cudaStream_t st,
                   const PUpdate *pu = nullptr);
void nufft_adjoint(NufftPlan &p, const float2 *samples, SampleLayout layout, const float *dcw, const float2 *csm,
                   int nb, float2 *img, bool img_os, bool accumulate, float weight, int fft_dir, cudaStream_t st);
void nufft_normal(NufftPlan &p, const float2 *img, const float2 *csm, int nb, const float *dcw, float2 *out,
                  bool accumulate, float weight, cudaStream_t st);
void nufft_compute(NufftPlan &p, const void *in, void *out, const float *dcw, gb_comp_mode mode, int nb,
                   bool image_os, cudaStream_t st);
void nufft_mult_MH_M(NufftPlan &p, const void *in, void *out, const float *dcw, int nb, cudaStream_t st);
void nufft_time_normal_convolutions(NufftPlan &p, int nb, const float *dcw, int reps, void *flush,
                                    size_t flush_bytes, float *ms_grid, float *ms_degrid, cudaStream_t st);
void nufft_convolve(NufftPlan &p, const void *in, void *out, gb_conv_mode mode, bool accumulate, int nb,
                    cudaStream_t st);
void nufft_fft(NufftPlan &p, void *data, gb_fft_mode mode, bool do_scale, int nbf, cudaStream_t st);
void nufft_deapodize(NufftPlan &p, void *data, int nbf, cudaStream_t st);
void nufft_traj_grad(NufftPlan &p, const float2 *img, const float2 *weights, const float *dcw, float *grad,
                     int nb, cudaStream_t st);
void nufft_traj_grad_from_grid(NufftPlan &p, const float2 *grid, const float2 *weights, float *grad, int nb,
                               cudaStream_t st);

// Cyclic k-space accumulation buffer (cuBuffer / cuSenseBuffer, gb_buffer.cu).
struct SenseBuffer {
    std::unique_ptr<NufftPlan> plan;
    int D = 0, coils = 0, cycle_length = 0, sub_cycle_length = 0;
    int cur_idx = 0, cur_sub_idx = 0;
    bool acc_empty = true;
    bool has_acc_image = false;   // the last accumulated coil images (reused by the combined image)
    const float *dcw = nullptr;   // retained
    const float2 *csm = nullptr;  // retained
    DevBuf<float2> acc, cyc, scaled, work, acc_image;
    void setup(int D, const uint64_t *N, const uint64_t *mos, float W, int coils, int num_cycles,
               int num_sub_cycles, cudaStream_t st);
    void clear(cudaStream_t st);
    bool add_frame_data(const float2 *samples, const float *traj, int64_t M, cudaStream_t st);
    void accumulated_coil_images(float2 *out, cudaStream_t st);
    void combined_coil_image(float2 *out, cudaStream_t st);
};

// Gridding with caller-provided scratch (no device allocation).
void grid_scratch_need(const NufftPlan &p, int nb, size_t *partial_elems, size_t *counter_elems);
void launch_grid_external_scratch(NufftPlan &p, const float2 *samples, float2 *grid, int nb, bool accumulate,
                                  float2 *partials, unsigned int *counters, cudaStream_t st);
// The plan behind a C handle (defined with the C ABI).
NufftPlan *plan_from_handle(gb_nufft_plan h);
// Status code (and error message) for the exception being handled.
gb_status current_exception_status();

// SENSE
void sense_mult_M(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st);
void sense_mult_MH(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st);
void sense_mult_MH_M(SenseOp &s, const void *in, void *out, bool accumulate, cudaStream_t st);

// CG
void cg_solve(CgSolver &cg, const void *d, void *x_out, double *hist, uint32_t *iters_run, cudaStream_t st);

}  // namespace gb
