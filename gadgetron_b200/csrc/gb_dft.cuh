// Register DFT machinery of the project-written FFT passes, shared by the
// pass kernels (gb_fft.cu) and the CG kernels that fuse a row pass with the
// pad or the crop (gb_ops.cu).  See gb_fft.cu for the algorithm.
#pragma once
#include <cstdint>
#include <type_traits>

#include "gb_internal.cuh"

namespace gb {

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

// Row transform of N = 16 N2 contiguous points by a half-warp (t = lane &
// 15 holds points t + 16 j): the N2-point register DFTs, the twiddles
// W_N^(t k2) (table tw), the exchange through rs (17 N2 float2 of this
// half-warp's shared memory, points padded by one every 16: conflict-free),
// then the 16-point DFTs give X[k2 + N2 q].  load(o) supplies input point o
// (called only inside the IN span), store(kk, v) takes output kk (only inside
// the OUT span).  Inverse (sg = -1) runs as conj(DFT(conj x)).  Both halves
// of the warp must call it (it has __syncwarp()s).  The first 16 columns'
// exchange cells (rs[0, 272)) are all read before the first store, and later
// groups read only above them: store may write there (a caller's output row
// of at most 272 points can share the exchange buffer).
template <int N2, int IN, int OUT, class Load, class Store>
__device__ __forceinline__ void row_fft_halfwarp(int t, float sg, const float2 *__restrict__ tw, float2 *rs,
                                                 int in_lo, int in_hi, int out_lo, int out_hi, Load load,
                                                 Store store) {
    constexpr int G = (N2 + 15) / 16;
    {
        float2 x[N2];
#pragma unroll
        for (int j = 0; j < N2; j++) {
            const int o = t + 16 * j;
            float2 v = make_float2(0.f, 0.f);
            if (in_span<IN, N2>(j, o, in_lo, in_hi)) v = load(o);
            x[j] = make_float2(v.x, sg * v.y);
        }
        dft<N2>(x);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            float2 y = x[k2];
            if (k2 > 0) y = cmul(y, __ldg(tw + t * k2));
            rs[t + 17 * k2] = y;   // point t + 16 k2 of the padded row
        }
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int k2 = t + 16 * g;
        float2 z[16];
        if (k2 < N2) {
#pragma unroll
            for (int u = 0; u < 16; u++) z[u] = rs[u + 17 * k2];
        }
        if (g == 0) __syncwarp();   // columns 0..15 read before any store
        if (k2 < N2) {
            dft<16>(z);
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int kk = k2 + N2 * q;
                if (out_span<OUT, N2>(q, kk, out_lo, out_hi)) store(kk, make_float2(z[q].x, sg * z[q].y));
            }
        }
    }
}

}  // namespace gb
