// Internal declarations shared by the gadgetron_b200 CUDA sources.
//
// Data layout in HBM (x fastest everywhere, as in the reference arrays):
//   image     [batches][frames][prod(N)]      complex64 (float2)
//   grid      [batches][frames][prod(mos)]    complex64  (oversampled, k-space)
//   samples   [batches][M_total]              complex64  (frame f owns
//                                                         [off[f], off[f+1]))
//   positions [D][M_total] float, sorted by tile ("home" order)
//
// The oversampled grid is cut into tiles of T_x x T_y x T_z cells.  Every
// sample has one home tile (the tile holding floor(s) - pad/2); the degridding
// kernel stages a home tile plus a halo of pad/2 cells and serves all its home
// samples.  The gridding kernel owns a tile exclusively (no atomics): its
// sample list holds every sample whose footprint touches the tile.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gadgetron_b200.h"

namespace gb {

constexpr int kMaxD = 3;
constexpr int kWMax = 8;          // max taps per dimension (W <= 7)
constexpr int kThreads = 256;     // threads per CTA for the tile kernels
constexpr int kChunk = 64;        // samples staged per pass (gridding)

// ------------------------------------------------------------ errors -----

struct Error {
    gb_status status;
    std::string msg;
};

void set_error(const std::string &msg);
// Counts kernel launches of this library (gb_kernel_launch_count).
void note_launch(uint64_t n = 1);
uint64_t launch_count();
[[noreturn]] void fail(gb_status st, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);
void check_cufft(cufftResult r, const char *what);

// A batch (or frame x batch) count taken from the C ABI as uint32_t and used
// as int: zero and values above INT_MAX are rejected before the conversion.
inline int count_arg(uint32_t v, const char *what) {
    if (v == 0 || v > 0x7fffffffu)
        fail(GB_ERR_INVALID_ARGUMENT, std::string(what) + " must be in [1, 2^31 - 1]");
    return static_cast<int>(v);
}

#define GB_CUDA(x) ::gb::check_cuda((x), #x)
#define GB_CUFFT(x) ::gb::check_cufft((x), #x)

// ------------------------------------------------- device buffer (RAII) ---

template <class T>
struct DevBuf {
    T *ptr = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
    // Grows to at least `count` elements; returns true if reallocated.
    bool ensure(size_t count) {
        if (count <= n && ptr) return false;
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)&ptr, count * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            fail(GB_ERR_OUT_OF_MEMORY, "device allocation of " +
                 std::to_string(count * sizeof(T)) + " bytes failed");
        }
        n = count;
        return true;
    }
    T *get() const { return ptr; }
};

// Preprocess sorting (gb_sort.cu): stable radix sort of (key, value) pairs by
// the low end_bit bits of the key, and an exclusive scan of n counts; both
// take their scratch from tmp (grown as needed).
void sort_pairs(const uint32_t *keys_in, uint32_t *keys_out, const uint32_t *vals_in, uint32_t *vals_out, int64_t n,
                int end_bit, DevBuf<unsigned char> &tmp, cudaStream_t st);
void exclusive_scan(const uint32_t *in, uint32_t *out, int64_t n, DevBuf<unsigned char> &tmp, cudaStream_t st);

// Scratch of a setup routine kept per device between calls (grown to the
// largest call, never shrunk): a struct S with a std::mutex `mu`, which a
// call holds until its stream is done with the scratch.  The cache is never
// destroyed; its device memory goes back with the context at exit.
template <class S>
S &device_scratch(int device) {
    static std::mutex map_mu;
    static auto *cache = new std::map<int, std::unique_ptr<S>>();
    std::lock_guard<std::mutex> lock(map_mu);
    auto &slot = (*cache)[device];
    if (!slot) slot.reset(new S());
    return *slot;
}

// --------------------------------------------------------- kernel params ---

// Plan constants passed by value to every kernel.
struct KParams {
    int D;
    int mos[kMaxD];        // oversampled size per dim (1 for unused dims)
    int N[kMaxD];          // matrix size per dim
    int tile[kMaxD];       // tile size per dim
    int ntiles[kMaxD];     // tiles per dim
    int hw;                // pad/2 = ceil(W/2)
    float radius;          // W/2
    float one_over_W;
    float beta[kMaxD];
    float mos_f[kMaxD];
    long long G;           // prod(mos)
    long long NN;          // prod(N)
    int ntiles_total;
};

// Address of cell (x, y, z) of batch bf = b*F + f in a k-space array:
//   bf*s_bf + z*s_z + y*s_y + x.
// Standard layout (every array a caller passes in): [bf][z][y][x].
// Outer-major layout (the plan's own oversampled workspaces, D >= 2): the
// outermost dimension (y in 2D, z in 3D) is moved in front of the batch,
// [y][bf][x] or [z][bf][y][x], so that the rows (2D) or slices (3D) of the
// N-wide interior band form one contiguous run over all batches and the FFT
// pass over the inner dimensions can skip the zero rows/slices.
struct KLayout {
    long long s_bf, s_y, s_z;
};

// One unit of tile work: frame*ntiles + tile, a range of a sample list and,
// for gridding tiles split across CTAs, the split bookkeeping.
struct WorkItem {
    int ft;        // frame * ntiles_total + tile
    int begin;     // range in the list
    int end;
    int split;     // -1: not split; else index into split table
    int chunk;     // chunk index within the split
    int pad0, pad1, pad2;
};

__host__ __device__ inline KLayout klayout_standard(const KParams &k) {
    KLayout l;
    l.s_bf = k.G;
    l.s_y = k.mos[0];
    l.s_z = (long long)k.mos[1] * k.mos[0];
    return l;
}

__host__ __device__ inline KLayout klayout_outer(const KParams &k, long long nbf) {
    KLayout l;
    if (k.D == 2) {
        l.s_bf = k.mos[0];
        l.s_y = nbf * k.mos[0];
        l.s_z = 0;
    } else if (k.D == 3) {
        l.s_bf = (long long)k.mos[1] * k.mos[0];
        l.s_y = k.mos[0];
        l.s_z = nbf * k.mos[1] * k.mos[0];
    } else {
        l = klayout_standard(k);
    }
    return l;
}

__host__ __device__ inline long long kaddr(const KLayout &l, long long bf, int x, int y, int z) {
    return bf * l.s_bf + z * l.s_z + y * l.s_y + x;
}

// Floats of the weight part of a pair row and of a whole pair row.
__host__ __device__ inline int pair_row_weights(const KParams &k) {
    return (k.tile[0] + k.tile[1] + (k.D == 3 ? k.tile[2] : 0) + 3) & ~3;
}
__host__ __device__ inline int pair_row_floats(const KParams &k) { return pair_row_weights(k) + 4; }

// Device-side scalars of one CG segment (a frame, or all frames).
struct CgSeg {
    double rq, rq0, alpha_re, alpha_im, beta, metric;
    int done, pad;
    unsigned int ctr_dot, ctr_upd, ctr_init, pad2;
};

// CG search-direction update folded into the forward pad of the normal
// operator: p = beta p + P^2 r for segments still running, done in place on
// the image being padded (p).  seg_per_frame: segment = frame, else one.
struct PUpdate {
    float2 *p;
    const float2 *r;
    const float *P;
    const CgSeg *segs;
    int seg_per_frame;
};

struct SplitInfo {
    int first_slot;  // first partial slot
    int nchunks;
};

// ----------------------------------------------------------- the plan -----

struct Tiling {
    int tile[kMaxD] = {16, 16, 1};
    int cg = 8;                 // coils per CTA (coil group)
    int split_len = 0;          // gridding list length above which a tile is split (0 = auto)
    int schedule = 0;           // E^H E gridding: 0 auto, 1 one CTA per work item, 2 persistent work queue
};

struct NufftPlan {
    int D = 0;
    int64_t N[kMaxD] = {1, 1, 1};
    int64_t mos[kMaxD] = {1, 1, 1};
    float W = 0.f;
    uint32_t flags = 0;
    int device = 0;
    KParams kp{};
    Tiling tiling;

    // preprocess state
    bool prepped = false;
    uint64_t generation = 0;       // bumped by every preprocess (invalidates captured graphs)
    DevBuf<float> traj_copy;       // the preprocessed trajectory (for re-binning)
    // preprocessing scratch, kept between calls (no allocation when sizes repeat)
    DevBuf<float> pp_pos;
    DevBuf<uint32_t> pp_key, pp_idx, pp_key_sorted, pp_counts, pp_pcnt, pp_poff, pp_pkey, pp_pval, pp_pkey_sorted;
    DevBuf<unsigned char> pp_sort;   // sort and scan scratch
    DevBuf<int64_t> pp_off;
    DevBuf<int> pp_err;
    // The two device segments of preprocess (before and after the pair count
    // is read back), recorded as CUDA graphs the second time the same shapes
    // arrive on the same buffers and replayed from then on (one launch
    // instead of ~20: preprocess runs in every end-to-end reconstruction).
    struct PrepGraph {
        cudaGraphExec_t exec = nullptr;
        uint64_t key = 0;       // shapes and buffers exec was recorded with
        uint64_t seen = 0;      // those of the last eager run
        uint64_t kernels = 0;   // kernels per replay (launch counter)
    } prep_graph[2];
    uint32_t *h_stage = nullptr;   // pinned host words for preprocess readbacks
    size_t h_stage_n = 0;
    unsigned char *h_upload = nullptr;   // pinned staging of preprocess uploads (frame offsets, work lists)
    size_t h_upload_n = 0;
    cudaEvent_t upload_done = nullptr;   // recorded after the last upload from h_upload
    gb_prep_mode prep_mode = GB_PREP_ALL;
    bool prepped_c2nc = false, prepped_nc2c = false;
    uint32_t F = 0;
    int64_t Mtot = 0;
    std::vector<int64_t> frame_off;
    DevBuf<float> pos_sorted;      // [D][Mtot]
    DevBuf<float> wtab;            // [Mtot][D][kWMax] 1D kernel weights of the taps of sorted samples
    DevBuf<uint32_t> perm;         // sorted pos -> original sample index
    DevBuf<uint32_t> home_off;     // [F*ntiles + 1]
    DevBuf<uint32_t> grid_list;    // gridding pair list (sorted positions)
    // Per gridding pair, the sample's 1D weights laid over the tile: rows of
    // pair_row_stride floats = x weights (tile x), y weights (tile y), z
    // weights (tile z, 3D), padding to a multiple of 4, then 4 words of the
    // tile-local footprint ranges (lo | hi << 16 per dimension).  Built at
    // preprocess for D >= 2 (pair_row_stride = 0 when not built).
    DevBuf<float> pair_rows;
    int pair_row_stride = 0;
    DevBuf<unsigned int> err_flag;   // set by kernels whose bounded waits ran out
    DevBuf<uint32_t> grid_off;     // [F*ntiles + 1]
    DevBuf<WorkItem> deg_items;
    int n_deg_items = 0;
    DevBuf<WorkItem> grd_items;
    int n_grd_items = 0;
    DevBuf<SplitInfo> splits;
    int n_splits = 0, n_slots = 0;
    DevBuf<unsigned int> split_counters;   // [n_splits * max coil groups]
    DevBuf<unsigned int> grid_queue;       // persistent gridding: next unit, CTAs finished (zero between launches)
    int split_counter_groups = 0;
    DevBuf<float2> partials;               // [n_slots][cg_groups][cells*cg]
    int64_t total_pairs = 0;
    std::vector<uint32_t> h_home_counts;   // per (frame, tile), for tuning

    // deapodization: per-dim reciprocal of the 1D kernel transform
    DevBuf<float> deap_img;   // [D][maxN]    1/psi_d(n + (mos-N)/2)
    DevBuf<float> deap_os;    // [D][maxmos]  1/psi_d(g)
    int maxN = 0, maxmos = 0;

    // workspaces
    DevBuf<float2> img_os;    // padded image, zero outside the interior
    size_t img_os_batches_zeroed = 0;
    bool img_os_dirty = true;
    int64_t img_os_nbf = -1;       // batch count whose outer-major band the pad buffer holds
    DevBuf<float2> kgrid;     // k-space grid
    DevBuf<float2> samp_ws;   // samples in tile order [batches][Mtot]
    std::map<int, cufftHandle> fft_plans;   // batch -> plan (standard layout, rank D)
    std::map<std::pair<int, int>, cufftHandle> fft_plans_om;   // (batch, pass) -> plan (outer-major)
    std::map<int, DevBuf<float2>> fft_tw;   // transform length -> W_N^e table (project-written passes)

    ~NufftPlan();
};

// ------------------------------------------------ host-side operations ----

void plan_init(NufftPlan &p, int D, const uint64_t *N, const uint64_t *mos, float W,
               uint32_t flags);
void plan_preprocess(NufftPlan &p, const float *traj, uint64_t Mtot, uint32_t F,
                     const uint64_t *frame_offsets, gb_prep_mode mode, cudaStream_t st);
void plan_build_work(NufftPlan &p, cudaStream_t st);
cufftHandle plan_fft(NufftPlan &p, int batches, cudaStream_t st);

// FFT passes over an outer-major workspace of nbf batches (D >= 2):
//   FFT_PASS_A_BAND / FFT_PASS_A_FULL: the inner dimensions (x in 2D, y-x
//     slices in 3D), over the N-wide band of the outer dimension or all of it;
//   FFT_PASS_B: the outer dimension (y in 2D, z in 3D), every column.
enum FftPass { FFT_PASS_A_BAND = 0, FFT_PASS_A_FULL = 1, FFT_PASS_B = 2 };
cufftHandle plan_fft_om(NufftPlan &p, int nbf, FftPass pass, cudaStream_t st);
// Element offset of the band start for FFT_PASS_A_BAND.
int64_t fft_band_offset(const NufftPlan &p, int nbf);

// Project-written FFT passes (gb_fft.cu), used instead of cuFFT for D >= 2
// when every oversampled size is 16 * n2 with n2 in {2, 4, 6, 8, 10, 12, 16,
// 20, 24, 32, 40}.  fft_cols: `ncols` columns (col / cpp = plane at
// plane * pstride, col % cpp = offset), points at o * ostride.  fft_rows:
// `nrows` rows of n contiguous points (row r at (r / rpp) * pstride +
// (row_off + r % rpp) * n).  Input points outside [in_lo, in_hi) are taken as
// zero without being read; only points in [out_lo, out_hi) are written.
bool fft_custom_ok(const NufftPlan &p);
// W_N^e, e < N, for the project FFT passes of length n (created on first use,
// outside any stream capture; synchronises then).
const float2 *fft_twiddles(NufftPlan &p, int n, cudaStream_t st);
void fft_custom_prepare(NufftPlan &p, cudaStream_t st);
void fft_cols(NufftPlan &p, int n, const float2 *in, float2 *out, int64_t ncols, int64_t cpp, int64_t pstride,
              int64_t ostride, int in_lo, int in_hi, int out_lo, int out_hi, bool inverse, cudaStream_t st);
void fft_rows(NufftPlan &p, int n, const float2 *in, float2 *out, int64_t nrows, int64_t rpp, int64_t row_off,
              int64_t pstride, int in_lo, int in_hi, int out_lo, int out_hi, bool inverse, cudaStream_t st);
void plan_set_tiling(NufftPlan &p, const int *tile, int cg);
// The tiling a new plan starts with (16 x 16 in 2D, 8^3 in 3D, coil group 16).
void plan_default_tiling(NufftPlan &p);
// Hash of every buffer address and count the convolution kernels' launches
// depend on: equal signatures mean a captured graph is still valid.
uint64_t plan_layout_signature(const NufftPlan &p, int nbf);
// Times candidate tilings on the preprocessed trajectory with `nb` batches and
// keeps the fastest (cached per workload key for later plans).
void plan_autotune(NufftPlan &p, int nb, cudaStream_t st);

// Sample-array layout flags for the convolution kernels.
//   ORIGINAL   [nb][Mtot], the caller's sample order
//   SORTED     [nb][Mtot], the plan's sorted (home tile) order
//   SORTED_IL  [Mtot][il] sorted order with the coils of a sample adjacent
//              (il = nb rounded up to even, so a sample's coil group is a
//              16-byte multiple): the plan's own workspace between
//              degridding and gridding inside E^H E, which the gridding
//              kernel stages by bulk copies (no gather through registers).
enum SampleLayout { LAYOUT_ORIGINAL = 0, LAYOUT_SORTED = 1, LAYOUT_SORTED_IL = 2 };
__host__ __device__ inline int il_stride_for(int nb) { return (nb + 1) & ~1; }
// The layout that E^H E hands from degridding to gridding for nb batches:
// SORTED_IL when the gridding runs the row variant (bulk-copied values),
// else SORTED.
SampleLayout normal_op_layout(const NufftPlan &p, int nb);

// Degridding: grid [nb][F][G] -> samples.  sign_fold multiplies the weight of
// grid cell g by (-1)^(sum g) (the centring checkerboard after the FFT).
// dcw (original sample order, may be null) multiplies the output, dcw_pow
// times (1 or 2).
void launch_degrid(NufftPlan &p, const float2 *grid, float2 *samples, int nb,
                   SampleLayout layout, const float *dcw, int dcw_pow, bool sign_fold,
                   bool accumulate, cudaStream_t st, const KLayout *kl = nullptr);

// Gridding: samples -> grid [nb][F][G] (overwritten unless accumulate).
// dcw multiplies the input samples (may be null).
void launch_grid(NufftPlan &p, const float2 *samples, float2 *grid, int nb,
                 SampleLayout layout, const float *dcw, bool sign_fold, bool accumulate,
                 cudaStream_t st, const KLayout *kl = nullptr);

// Trajectory gradient from a k-space grid (sign folded like the degridder).
void launch_traj_grad(NufftPlan &p, const float2 *grid, const float2 *weights, int nb,
                      const float *dcw, float *grad, bool sign_fold, cudaStream_t st,
                      const KLayout *kl = nullptr);

// Image-side fused kernels.
// Forward: dst_os[b][f][interior] = src[...] * (csm) * deap * sign * scale.
//   csm == null: src [nb][F][NN] -> dst [nb][F][G]
//   csm != null: src [F][NN], csm [C][NN] -> dst [C][F][G] (nb = C)
// With an outer-major dst (D >= 2) the whole rows/slices of the interior band
// are written (zeros outside the interior), so an in-place FFT pass over the
// band may follow; the rest of dst must already be zero.
// pu (optional, csm path only): the CG direction update applied to src first.
void launch_pad_forward(NufftPlan &p, const float2 *src, const float2 *csm, float2 *dst,
                        int nb, bool src_oversampled, cudaStream_t st, const KLayout *kl = nullptr,
                        const PUpdate *pu = nullptr);
// Adjoint: dst[...] (+)= crop(grid) * deap * sign * scale (* conj(csm) summed over coils)
//   csm == null: grid [nb][F][G] -> dst [nb][F][NN] (or [nb][F][G] when dst_oversampled)
//   csm != null: grid [C][F][G] -> dst [F][NN]
void launch_crop_adjoint(NufftPlan &p, const float2 *grid, const float2 *csm, float2 *dst,
                         int nb, bool dst_oversampled, bool accumulate, float weight,
                         bool fourier_deapod, cudaStream_t st, const KLayout *kl = nullptr);

// Reference-form utilities (NFFT_plan::fft / deapodize on oversampled arrays).
void launch_timeswitch_scale(NufftPlan &p, float2 *data, int nbf, float scale, cudaStream_t st);
void launch_deapodize_os(NufftPlan &p, float2 *data, int nbf, cudaStream_t st);
void launch_multiply_dcw(const float *dcw, float2 *data, int64_t M, int nb, cudaStream_t st);

// ------------------------------------------------------- device helpers ---

__host__ __device__ __forceinline__ float bessi0f_ref(float x) {
    // Rational approximation of I0 used by the reference kernel
    // (toolboxes/nfft/ConvolutionKernel.hpp:39-68), same coefficients and
    // evaluation order.
    if (x == 0.0f) return 1.0f;
    float z = x * x;
    float numerator = (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z *
                       (z * 0.210580722890567e-22f + 0.380715242345326e-19f) +
                       0.479440257548300e-16f) + 0.435125971262668e-13f) +
                       0.300931127112960e-10f) + 0.160224679395361e-7f) +
                       0.654858370096785e-5f) + 0.202591084143397e-2f) +
                       0.463076284721000e0f) + 0.754337328948189e2f) +
                       0.830792541809429e4f) + 0.571661130563785e6f) +
                       0.216415572361227e8f) + 0.356644482244025e9f) +
                       0.144048298227235e10f);
    float denominator = (z * (z * (z - 0.307646912682801e4f) + 0.347626332405882e7f) -
                         0.144048298227235e10f);
    return -numerator / denominator;
}

// d/dz of the rational function R(z) = -num(z)/den(z) that bessi0f_ref
// evaluates at z = x^2 (derivative of the same approximation, so finite
// differences of the forward operator agree with it).
__host__ __device__ __forceinline__ float bessi0_dRdz(float z) {
    const float a[15] = {0.144048298227235e10f, 0.356644482244025e9f, 0.216415572361227e8f,
                         0.571661130563785e6f,  0.830792541809429e4f, 0.754337328948189e2f,
                         0.463076284721000e0f,  0.202591084143397e-2f, 0.654858370096785e-5f,
                         0.160224679395361e-7f, 0.300931127112960e-10f, 0.435125971262668e-13f,
                         0.479440257548300e-16f, 0.380715242345326e-19f, 0.210580722890567e-22f};
    float num = a[14], dnum = 0.f;
    for (int i = 13; i >= 0; --i) {
        dnum = dnum * z + num;
        num = num * z + a[i];
    }
    // den(z) = z^3 - 3076.46912682801 z^2 + 3476263.32405882 z - 1.44048298227235e9
    const float b2 = -0.307646912682801e4f, b1 = 0.347626332405882e7f, b0 = -0.144048298227235e10f;
    float den = ((z + b2) * z + b1) * z + b0;
    float dden = (3.f * z + 2.f * b2) * z + b1;
    // R = -num/den ; R' = -(num' den - num den') / den^2
    return -(dnum * den - num * dden) / (den * den);
}

// One-dimensional Kaiser-Bessel value in the reference's arithmetic
// (toolboxes/nfft/ConvolutionKernel.hpp:85-94), zero beyond the radius
// (ConvolutionKernel.hpp:164-170).  Non-finite values are returned as 0: the
// reference drops a tap whose product weight is not finite
// (ConvolverC2NC.cuh:96-97, ConvolverNC2C_standard.cuh:266-268).
__device__ __forceinline__ float kb_weight_1d(float delta, float mos_f, float one_over_W,
                                              float beta, float radius) {
    if (delta > radius) return 0.f;
    float _tmp = 2.0f * delta * one_over_W;
    float tmp = _tmp * _tmp;
    float arg = beta * sqrtf(1.0f - tmp);
    float bessi = bessi0f_ref(arg);
    float w = mos_f * bessi * one_over_W;
    return isfinite(w) ? w : 0.f;
}

// d/d(delta) of the 1D kernel for delta in [0, radius]:
//   phi(u) = mos/W * R(beta^2 (1 - (2u/W)^2))
//   phi'(u) = -(8 mos beta^2 u / W^3) * R'(z)
__device__ __forceinline__ float kb_deriv_1d(float delta, float mos_f, float one_over_W,
                                             float beta, float radius) {
    if (delta > radius) return 0.f;
    float t = 2.0f * delta * one_over_W;
    float z = beta * beta * (1.0f - t * t);
    if (!(z >= 0.f)) return 0.f;
    float ow3 = one_over_W * one_over_W * one_over_W;
    float d = -8.0f * mos_f * beta * beta * delta * ow3 * bessi0_dRdz(z);
    return isfinite(d) ? d : 0.f;
}

__host__ __device__ __forceinline__ int wrapmod(int x, int m) {
    int r = x % m;
    return r < 0 ? r + m : r;
}

// Image regulariser and preconditioner weights (gb_reg.cu).  Returns the
// offset; image receives 1 / (|reg n / asum(reg)| + offset).
float image_operator_compute(const float2 *reg, int64_t n, bool offset_estimation, float *image,
                             cudaStream_t st);
// w = 1 / sqrt(sum_c |csm_c|^2 + kappa * reg) over nn pixels (reg may be null).
void sense_precond_weights(const float2 *csm, int nb, int64_t nn, const float *reg, float kappa, float *w,
                           cudaStream_t st);

// Radial trajectories [frames][profiles * S][2] and density compensation
// weights [profiles * S] (gb_radial.cu).
void radial_traj_golden(float *traj, int S, int P, int F, int profile_offset, int mode, cudaStream_t st);
void radial_traj_fixed(float *traj, int S, int P, int F, float angular_offset, cudaStream_t st);
void radial_traj_variable(float *traj, const float *angles, int S, int P, int F, cudaStream_t st);
void radial_dcw(float *dcw, int S, int P, float alpha, float ovs, int profile_offset, bool golden, int mode,
                cudaStream_t st);

// Iterative density compensation with a Jinc kernel (gb_sdc.cu).
void sdc_estimate_dcw(int D, const uint64_t *N, float os_factor, int iterations, float kernel_width,
                      const float *traj, int64_t M, const float *initial, float *dcw, cudaStream_t st);

// Coil sensitivity estimation from coil images [ncoils][dims] (gb_b1map.cu).
void estimate_b1_map(int D, const uint64_t *dims, int ncoils, int target_coils, const float2 *images, float2 *csm,
                     cudaStream_t st);

}  // namespace gb
