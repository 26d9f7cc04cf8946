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

constexpr double kTwoPi = 6.283185307179586476925;

// Compile-time cos(2 pi a / b) and sin(2 pi a / b) for the register DFTs'
// twiddles: the argument is reduced to [0, pi/4] by the symmetries of the
// circle (exact integer arithmetic on a / b), then a Taylor series in double.
__host__ __device__ constexpr double cx_sin_red(double x) {
    double x2 = x * x, term = x, sum = x;
    for (int n = 1; n <= 12; n++) {
        term *= -x2 / (double)((2 * n) * (2 * n + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cx_cos_red(double x) {
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int n = 1; n <= 12; n++) {
        term *= -x2 / (double)((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cx_cos2pi(long long a, long long b) {
    a %= b;
    if (a < 0) a += b;
    if (2 * a > b) a = b - a;              // cos(2 pi f) = cos(2 pi (1 - f)), f <= 1/2
    double sign = 1.0;
    if (4 * a > b) {                       // f in (1/4, 1/2]: cos = -cos(2 pi (1/2 - f))
        a = b - 2 * a;
        b = 2 * b;
        sign = -1.0;
    }
    // f = a / b in [0, 1/4]
    if (8 * a > b) return sign * cx_sin_red(6.283185307179586476925 * (double)(b - 4 * a) / (double)(4 * b));
    return sign * cx_cos_red(6.283185307179586476925 * (double)a / (double)b);
}
__host__ __device__ constexpr double cx_sin2pi(long long a, long long b) {
    return cx_cos2pi(b - 4 * a, 4 * b);    // sin(2 pi f) = cos(2 pi (1/4 - f))
}

template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// -i * a
__device__ __forceinline__ float2 cmi(float2 a) { return make_float2(a.y, -a.x); }

// v * W_L^E with W_L = exp(-2 pi i / L) a compile-time constant; the
// multiples of 1/8 turn are additions and sign changes.
template <int L, int E>
__device__ __forceinline__ float2 tw_mul(float2 v) {
    constexpr int e = E % L;
    constexpr float h = 0.70710678118654752440f;   // sqrt(1/2)
    if constexpr (e == 0) {
        return v;
    } else if constexpr (4 * e == L) {
        return cmi(v);
    } else if constexpr (2 * e == L) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * e == 3 * L) {
        return make_float2(-v.y, v.x);
    } else if constexpr (8 * e == L) {
        return make_float2(h * (v.x + v.y), h * (v.y - v.x));
    } else if constexpr (8 * e == 3 * L) {
        return make_float2(h * (v.y - v.x), -h * (v.x + v.y));
    } else {
        constexpr float c = (float)cx_cos2pi(e, L), sn = (float)(-cx_sin2pi(e, L));
        return make_float2(v.x * c - v.y * sn, v.x * sn + v.y * c);
    }
}

// In-place forward DFT of N points in registers (natural order in and out).
template <int N>
__device__ __forceinline__ void dft(float2 (&x)[N]) {
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        const float2 a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    } else if constexpr (N == 3) {
        constexpr float h = 0.86602540378443864676f;   // sin(2 pi / 3)
        const float2 a = x[0], s = cadd(x[1], x[2]), d = csub(x[1], x[2]);
        const float2 m = make_float2(a.x - 0.5f * s.x, a.y - 0.5f * s.y);
        x[0] = cadd(a, s);
        x[1] = make_float2(m.x + h * d.y, m.y - h * d.x);
        x[2] = make_float2(m.x - h * d.y, m.y + h * d.x);
    } else if constexpr (N == 4) {
        const float2 s0 = cadd(x[0], x[2]), d0 = csub(x[0], x[2]);
        const float2 s1 = cadd(x[1], x[3]), d1 = cmi(csub(x[1], x[3]));
        x[0] = cadd(s0, s1);
        x[2] = csub(s0, s1);
        x[1] = cadd(d0, d1);
        x[3] = csub(d0, d1);
    } else if constexpr (N == 5) {
        constexpr float c1 = 0.30901699437494742410f;    // cos(2 pi / 5)
        constexpr float c2 = -0.80901699437494742410f;   // cos(4 pi / 5)
        constexpr float s1 = 0.95105651629515357212f;    // sin(2 pi / 5)
        constexpr float s2 = 0.58778525229247312917f;    // sin(4 pi / 5)
        const float2 a = x[0];
        const float2 sa = cadd(x[1], x[4]), da = csub(x[1], x[4]);
        const float2 sb = cadd(x[2], x[3]), db = csub(x[2], x[3]);
        const float2 m1 = make_float2(a.x + c1 * sa.x + c2 * sb.x, a.y + c1 * sa.y + c2 * sb.y);
        const float2 m2 = make_float2(a.x + c2 * sa.x + c1 * sb.x, a.y + c2 * sa.y + c1 * sb.y);
        const float2 n1 = make_float2(s1 * da.x + s2 * db.x, s1 * da.y + s2 * db.y);
        const float2 n2 = make_float2(s2 * da.x - s1 * db.x, s2 * da.y - s1 * db.y);
        x[0] = make_float2(a.x + sa.x + sb.x, a.y + sa.y + sb.y);
        x[1] = cadd(m1, cmi(n1));
        x[4] = csub(m1, cmi(n1));
        x[2] = cadd(m2, cmi(n2));
        x[3] = csub(m2, cmi(n2));
    } else {
        constexpr int R = (N % 4 == 0) ? 4 : (N % 2 == 0 ? 2 : (N % 3 == 0 ? 3 : 5));
        constexpr int M = N / R;
        static_assert(R * M == N, "unsupported register DFT size");
        float2 s[R][M];
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int m = 0; m < M; m++) s[r][m] = x[m * R + r];
#pragma unroll
        for (int r = 0; r < R; r++) dft<M>(s[r]);
        static_for<0, M>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            float2 t[R];
            static_for<0, R>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                t[r] = tw_mul<N, r * k>(s[r][k]);
            });
            dft<R>(t);
#pragma unroll
            for (int q = 0; q < R; q++) x[k + M * q] = t[q];
        });
    }
}

// Which points a pass reads (IN) or writes (OUT): all of them, the centred
// half [N/4, 3N/4) (alpha = 2; known at compile time, so the zero inputs and
// the unused outputs drop out of the register DFTs), or a runtime range.
enum : int { kSpanAll = 0, kSpanHalf = 1, kSpanRange = 2 };

// Input point o = t + 16 j (t < 16 at run time, j unrolled).
template <int SPAN, int N2>
__device__ __forceinline__ bool in_span(int j, int o, int lo, int hi) {
    if constexpr (SPAN == kSpanAll) {
        return true;
    } else if constexpr (SPAN == kSpanHalf && N2 % 4 == 0) {
        return j >= N2 / 4 && j < 3 * N2 / 4;   // [4 N2, 12 N2) = whole groups of 16
    } else if constexpr (SPAN == kSpanHalf) {
        return o >= 4 * N2 && o < 12 * N2;
    } else {
        return o >= lo && o < hi;
    }
}
// Output point kk = k2 + N2 q (k2 < N2 at run time, q < 16 unrolled).
template <int SPAN, int N2>
__device__ __forceinline__ bool out_span(int q, int kk, int lo, int hi) {
    if constexpr (SPAN == kSpanAll) return true;
    else if constexpr (SPAN == kSpanHalf) return q >= 4 && q < 12;
    else return kk >= lo && kk < hi;
}

// Strided pass: column `col` (col / cpp = plane, col % cpp = offset in the
// plane) has its N points at base + o * ostride.  kColsPerCta adjacent
// columns per CTA, 16 threads per column; every load and store instruction of
// a warp covers four 64-byte runs.  Shared memory: N2 rows of kColsRow float2
// (16 t x 8 columns, padded so that the four t of a warp fall into two bank
// halves).
constexpr int kColsPerCta = 8;
constexpr int kColsRow = 16 * kColsPerCta + 8;

template <int N2, int IN, int OUT>
__global__ void __launch_bounds__(16 * kColsPerCta, 4) k_fft_cols(FftColArgs a) {
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
    constexpr int G = (N2 + 15) / 16;
    extern __shared__ float2 fft_sm[];
    const int r = threadIdx.x >> 4, t = threadIdx.x & 15;
    const int64_t gr = (int64_t)blockIdx.x * kRowsPerCta + r;
    const bool row_ok = gr < a.nrows;
    const int64_t pl = gr / a.rpp;
    const int64_t rbase = pl * a.pstride + (a.row_off + (gr - pl * a.rpp)) * (int64_t)N;
    const float sg = a.inverse ? -1.f : 1.f;
    float2 *rs = fft_sm + r * (17 * N2);
    {
        float2 x[N2];
#pragma unroll
        for (int j = 0; j < N2; j++) {
            const int o = t + 16 * j;
            float2 v = make_float2(0.f, 0.f);
            if (row_ok && in_span<IN, N2>(j, o, a.in_lo, a.in_hi)) v = a.in[rbase + o];
            x[j] = make_float2(v.x, sg * v.y);
        }
        dft<N2>(x);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            float2 y = x[k2];
            if (k2 > 0) y = cmul(y, __ldg(a.tw + t * k2));
            rs[t + 17 * k2] = y;   // point t + 16 k2 of the padded row
        }
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int k2 = t + 16 * g;
        if (k2 < N2) {
            float2 z[16];
#pragma unroll
            for (int u = 0; u < 16; u++) z[u] = rs[u + 17 * k2];
            dft<16>(z);
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int kk = k2 + N2 * q;
                if (row_ok && out_span<OUT, N2>(q, kk, a.out_lo, a.out_hi))
                    a.out[rbase + kk] = make_float2(z[q].x, sg * z[q].y);
            }
        }
    }
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
static const float2 *twiddles(NufftPlan &p, int n, cudaStream_t st) {
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
    for (int d = 0; d < p.D; d++) twiddles(p, p.kp.mos[d], st);
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
    FftColArgs a{in, out, cpp, pstride, ostride, in_lo, in_hi, out_lo, out_hi, inverse ? 1 : 0, twiddles(p, n, st)};
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
                 twiddles(p, n, st)};
    const int si = span_of(in_lo, in_hi, n), so = span_of(out_lo, out_hi, n);
#define GB_FFT_ROWS(K) launch_rows_n<K>(a, si, so, st)
    GB_FFT_N2_SWITCH(n / 16, GB_FFT_ROWS)
#undef GB_FFT_ROWS
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb
