// Batched complex FFTs of the oversampled workspaces (D >= 2).
//
// The reference runs cuFFT over the whole oversampled grid of every coil
// (cuNDFFT.cpp:110-142) between the pad and the gridding.  Here the two
// passes of each direction are project-written kernels over the outer-major
// workspace ([y][batch][x] in 2D, [z][batch][y][x] in 3D), which know which
// rows are zero or unused:
//   * forward: the padded image is zero outside the centred N band, so the
//     x pass reads only the band's columns and the outer pass reads only the
//     band's rows (half of each pass's input at alpha = 2);
//   * adjoint: the crop keeps only the centred band, so the outer pass writes
//     only the band's rows and the x pass only the band's columns.
// Transforms are unscaled (the 1/sqrt(G) is applied by the pad and the crop),
// forward = exp(-2 pi i k n / N), inverse = exp(+2 pi i k n / N) (the inverse
// runs as conj(DFT(conj(x)))).
//
// Algorithm: N = 16 * N2 (N2 = 2..40, even, with factors 2, 3, 5).  Point o = t + 16 j
// (t < 16, j < N2).  Thread t of a column (or row) does the N2-point DFT of its
// points in registers, multiplies by W_N^(t k2), and after an exchange through
// shared memory the 16-point DFTs over t give X[k2 + N2 q].  The register DFTs
// are mixed-radix decimation in time (radix 4, 2, 3, 5), fully unrolled, with
// compile-time twiddles.
#include <cmath>
#include <type_traits>
#include <vector>

#include "gb_dft.cuh"
#include "gb_internal.cuh"

namespace gb {

struct FftColArgs {
    const float2 *in;
    float2 *out;
    int64_t cpp, pstride, ostride;
    int in_lo, in_hi, out_lo, out_hi;
    int inverse;
    const float2 *tw;   // W_N^e, e < N
};

struct FftRowArgs {
    const float2 *in;
    float2 *out;
    int64_t nrows, rpp, row_off, pstride;
    int in_lo, in_hi, out_lo, out_hi;
    int inverse;
    const float2 *tw;
};

// Strided pass: column `col` (col / cpp = plane, col % cpp = offset in the
// plane) has its N points at base + o * ostride.  kColsPerCta adjacent
// columns per CTA, 16 threads per column; every load and store instruction of
// a warp covers four 64-byte runs.  Shared memory: N2 rows of kColsRow float2
// (16 t x 8 columns, padded so that the four t of a warp fall into two bank
// halves).
constexpr int kColsPerCta = 8;
constexpr int kColsRow = 16 * kColsPerCta + 8;

template <int N2, int IN, int OUT>
__global__ void __launch_bounds__(16 * kColsPerCta, (N2 <= 24) ? 6 : 4) k_fft_cols(FftColArgs a) {
    constexpr int N = 16 * N2;
    extern __shared__ float2 fft_sm[];
    const int c = threadIdx.x % kColsPerCta, t = threadIdx.x / kColsPerCta;
    const int64_t col = (int64_t)blockIdx.x * kColsPerCta + c;
    const int64_t plane = col / a.cpp;
    const int64_t base = plane * a.pstride + (col - plane * a.cpp);
    const float sg = a.inverse ? -1.f : 1.f;
    float2 x[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) {
        const int o = t + 16 * j;
        float2 v = make_float2(0.f, 0.f);
        if (in_span<IN, N2>(j, o, a.in_lo, a.in_hi)) v = a.in[base + (int64_t)o * a.ostride];
        x[j] = make_float2(v.x, sg * v.y);
    }
    dft<N2>(x);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) {
        float2 y = x[k2];
        if (k2 > 0) y = cmul(y, __ldg(a.tw + t * k2));
        fft_sm[k2 * kColsRow + t * kColsPerCta + c] = y;
    }
    __syncthreads();
    for (int k2 = t; k2 < N2; k2 += 16) {
        float2 z[16];
#pragma unroll
        for (int u = 0; u < 16; u++) z[u] = fft_sm[k2 * kColsRow + u * kColsPerCta + c];
        dft<16>(z);
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int kk = k2 + N2 * q;
            if (out_span<OUT, N2>(q, kk, a.out_lo, a.out_hi))
                a.out[base + (int64_t)kk * a.ostride] = make_float2(z[q].x, sg * z[q].y);
        }
    }
    (void)N;
}

// Contiguous pass: row r (r / rpp = plane, row_off + r % rpp = row in the
// plane) holds N contiguous points.  kRowsPerCta rows per CTA, 16 threads per
// row (a half-warp): thread t loads points t + 16 j straight from global memory
// (each load instruction covers two 128-byte runs), the exchange between the
// two DFT steps stays inside the half-warp (shared memory, rows padded by one
// float2 every 16 points: conflict-free), and the outputs X[k2 + N2 q] are
// stored straight to global memory (again 128-byte runs).
constexpr int kRowsPerCta = 4;

template <int N2, int IN, int OUT>
__global__ void __launch_bounds__(16 * kRowsPerCta, 8) k_fft_rows(FftRowArgs a) {
    constexpr int N = 16 * N2;
    extern __shared__ float2 fft_sm[];
    const int r = threadIdx.x >> 4, t = threadIdx.x & 15;
    const int64_t gr = (int64_t)blockIdx.x * kRowsPerCta + r;
    const bool row_ok = gr < a.nrows;
    const int64_t pl = gr / a.rpp;
    const int64_t rbase = pl * a.pstride + (a.row_off + (gr - pl * a.rpp)) * (int64_t)N;
    const float sg = a.inverse ? -1.f : 1.f;
    float2 *rs = fft_sm + r * (17 * N2);
    row_fft_halfwarp<N2, IN, OUT>(
        t, sg, a.tw, rs, a.in_lo, a.in_hi, a.out_lo, a.out_hi,
        [&](int o) { return row_ok ? a.in[rbase + o] : make_float2(0.f, 0.f); },
        [&](int kk, float2 v) {
            if (row_ok) a.out[rbase + kk] = v;
        });
    (void)N;
}

// ------------------------------------------------------------- host -----

static bool fft_len_ok(int n) {
    if (n % 16) return false;
    const int n2 = n / 16;
    switch (n2) {
        case 2: case 4: case 6: case 8: case 10: case 12: case 16: case 20: case 24: case 32: case 40:
            return true;
        default:
            return false;
    }
}

bool fft_custom_ok(const NufftPlan &p) {
    if (p.D < 2) return false;
    for (int d = 0; d < p.D; d++)
        if (!fft_len_ok(p.kp.mos[d])) return false;
    return true;
}

// W_N^e, e < N, for one transform length (device table owned by the plan).
const float2 *fft_twiddles(NufftPlan &p, int n, cudaStream_t st) {
    auto it = p.fft_tw.find(n);
    if (it != p.fft_tw.end()) return it->second.get();
    std::vector<float2> h(n);
    for (int e = 0; e < n; e++) {
        const double ang = kTwoPi * (double)e / (double)n;
        h[e] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
    }
    DevBuf<float2> &b = p.fft_tw[n];
    b.ensure(n);
    GB_CUDA(cudaMemcpyAsync(b.get(), h.data(), n * sizeof(float2), cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaStreamSynchronize(st));
    return b.get();
}

// Creates the twiddle tables the custom passes of this plan need (outside
// any stream capture).
void fft_custom_prepare(NufftPlan &p, cudaStream_t st) {
    if (!fft_custom_ok(p)) return;
    for (int d = 0; d < p.D; d++) fft_twiddles(p, p.kp.mos[d], st);
}

static int span_of(int lo, int hi, int n) {
    if (lo <= 0 && hi >= n) return kSpanAll;
    if (n % 4 == 0 && lo == n / 4 && hi == 3 * n / 4) return kSpanHalf;
    return kSpanRange;
}

template <int N2, int IN, int OUT>
static void launch_cols_m(const FftColArgs &a, int64_t ncols, cudaStream_t st) {
    const size_t smem = (size_t)N2 * kColsRow * sizeof(float2);
    auto kern = k_fft_cols<N2, IN, OUT>;
    if (smem > 48 * 1024) GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)(ncols / kColsPerCta), 16 * kColsPerCta, smem, st>>>(a);
    note_launch();
}

template <int N2, int IN, int OUT>
static void launch_rows_m(const FftRowArgs &a, cudaStream_t st) {
    const size_t smem = (size_t)kRowsPerCta * 17 * N2 * sizeof(float2);
    auto kern = k_fft_rows<N2, IN, OUT>;
    if (smem > 48 * 1024) GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)((a.nrows + kRowsPerCta - 1) / kRowsPerCta), 16 * kRowsPerCta, smem, st>>>(a);
    note_launch();
}

// The span combinations the workspace transforms use: a pruned input with
// every output (forward), every input with a pruned output (adjoint), both
// full; anything else runs with runtime ranges on both sides.
#define GB_FFT_SPAN_SWITCH(LAUNCH, N2, ...)                                              \
    do {                                                                                 \
        if (si == kSpanAll && so == kSpanAll) LAUNCH<N2, kSpanAll, kSpanAll>(__VA_ARGS__);          \
        else if (si == kSpanHalf && so == kSpanAll) LAUNCH<N2, kSpanHalf, kSpanAll>(__VA_ARGS__);   \
        else if (si == kSpanRange && so == kSpanAll) LAUNCH<N2, kSpanRange, kSpanAll>(__VA_ARGS__); \
        else if (si == kSpanAll && so == kSpanHalf) LAUNCH<N2, kSpanAll, kSpanHalf>(__VA_ARGS__);   \
        else if (si == kSpanAll && so == kSpanRange) LAUNCH<N2, kSpanAll, kSpanRange>(__VA_ARGS__); \
        else LAUNCH<N2, kSpanRange, kSpanRange>(__VA_ARGS__);                           \
    } while (0)

template <int N2>
static void launch_cols_n(const FftColArgs &a, int64_t ncols, int si, int so, cudaStream_t st) {
    GB_FFT_SPAN_SWITCH(launch_cols_m, N2, a, ncols, st);
}

template <int N2>
static void launch_rows_n(const FftRowArgs &a, int si, int so, cudaStream_t st) {
    GB_FFT_SPAN_SWITCH(launch_rows_m, N2, a, st);
}

#define GB_FFT_N2_SWITCH(n2, CALL)                  \
    switch (n2) {                                   \
        case 2: CALL(2); break;                     \
        case 4: CALL(4); break;                     \
        case 6: CALL(6); break;                     \
        case 8: CALL(8); break;                     \
        case 10: CALL(10); break;                   \
        case 12: CALL(12); break;                   \
        case 16: CALL(16); break;                   \
        case 20: CALL(20); break;                   \
        case 24: CALL(24); break;                   \
        case 32: CALL(32); break;                   \
        case 40: CALL(40); break;                   \
        default: fail(GB_ERR_INTERNAL, "unsupported FFT length"); \
    }

// Strided pass over `ncols` columns of length n (see k_fft_cols).
void fft_cols(NufftPlan &p, int n, const float2 *in, float2 *out, int64_t ncols, int64_t cpp, int64_t pstride,
              int64_t ostride, int in_lo, int in_hi, int out_lo, int out_hi, bool inverse, cudaStream_t st) {
    if (ncols % kColsPerCta || cpp % kColsPerCta) fail(GB_ERR_INTERNAL, "FFT column count must be a multiple of 8");
    if (ncols == 0) return;
    FftColArgs a{in, out, cpp, pstride, ostride, in_lo, in_hi, out_lo, out_hi, inverse ? 1 : 0, fft_twiddles(p, n, st)};
    const int si = span_of(in_lo, in_hi, n), so = span_of(out_lo, out_hi, n);
#define GB_FFT_COLS(K) launch_cols_n<K>(a, ncols, si, so, st)
    GB_FFT_N2_SWITCH(n / 16, GB_FFT_COLS)
#undef GB_FFT_COLS
    GB_CUDA(cudaGetLastError());
}

// Contiguous pass over `nrows` rows of length n (see k_fft_rows).
void fft_rows(NufftPlan &p, int n, const float2 *in, float2 *out, int64_t nrows, int64_t rpp, int64_t row_off,
              int64_t pstride, int in_lo, int in_hi, int out_lo, int out_hi, bool inverse, cudaStream_t st) {
    if (nrows == 0) return;
    FftRowArgs a{in, out, nrows, rpp, row_off, pstride, in_lo, in_hi, out_lo, out_hi, inverse ? 1 : 0,
                 fft_twiddles(p, n, st)};
    const int si = span_of(in_lo, in_hi, n), so = span_of(out_lo, out_hi, n);
#define GB_FFT_ROWS(K) launch_rows_n<K>(a, si, so, st)
    GB_FFT_N2_SWITCH(n / 16, GB_FFT_ROWS)
#undef GB_FFT_ROWS
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
