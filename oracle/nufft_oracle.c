/*
 * CPU oracle for the non-Cartesian NUFFT path (test infrastructure only).
 *
 * This file restates, in plain C, the arithmetic of the reference GPU NUFFT
 * (Gadgetron cuNFFT, STANDARD convolution).  It is the checker for the CUDA
 * library in gadgetron_b200/: only tests, the smoke check and the CPU
 * baseline leg of the benchmark load it.  Nothing in the product calls it.
 *
 * What follows the reference, and where:
 *   - bessi0 (float rational approximation):  toolboxes/nfft/ConvolutionKernel.hpp:39-68
 *   - KaiserBessel 1D value:                   toolboxes/nfft/ConvolutionKernel.hpp:85-94
 *   - separable product over dimensions:       toolboxes/nfft/ConvolutionKernel.hpp:108-130
 *   - get(): zero outside the radius (weak_greater, per dimension):
 *                                              toolboxes/nfft/ConvolutionKernel.hpp:164-170,
 *                                              toolboxes/core/vector_td_operators.h:309-313
 *   - beta (Beatty 2005):                      toolboxes/nfft/ConvolutionKernel.hpp:286-303
 *   - trajectory scaling k*mos + (mos+pad)/2:  toolboxes/nfft/gpu/ConvolverNC2C_standard.cuh:25-39,
 *                                              toolboxes/nfft/gpu/cuGriddingConvolution.cu:160-172
 *   - padding = 2*ceil(W/2):                   toolboxes/nfft/gpu/cuGriddingConvolution.cu:82-85
 *   - NC2C taps [ceil(s-W/2), floor(s+W/2)] on the padded grid, then the
 *     periodic wrap of the padding ring:       toolboxes/nfft/gpu/ConvolverNC2C_standard.cuh:41-102,229-292,358-477
 *   - C2NC taps on the unpadded grid with wrap: toolboxes/nfft/gpu/ConvolverC2NC.cuh:68-122,228-254
 *   - deapodization kernel image (a sample at mos/2):
 *                                              toolboxes/nfft/gpu/cuNFFT.cu:136-164
 *
 * Parity status: pinned against the reference's own outputs.  The
 * reference's GPU path (cuNFFT, cuNonCartesianSenseOperator, cuCgSolver) is
 * built from its sources into oracle/_ref/libgbref.so (oracle/build_ref.py)
 * and tests/test_ref_parity_gpu.py checks this restatement against it on the
 * same seeded inputs (relative L2 <= 1e-5), besides the known-answer case of
 * the reference's cuNFFT test, norm preservation of the centred FFT, the FP64
 * direct NDFT and exact adjointness (tests/test_known_answers.py,
 * tests/test_oracle.py).
 *
 * Fold of the padding ring (gridding, NC2C).  By default the ring is folded
 * periodically: every tap lands on its cell modulo mos, once.  That is what
 * the reference computes in 1D and 2D.  In 3D the reference's
 * wrap_image_kernel (ConvolverNC2C_standard.cuh:394-437) selects the
 * dimensions of each wrap combination with `i & combination` for i = 1..D,
 * which for i = 3 tests bits 0|1 instead of bit 2: on cells within the ring
 * width of a z face some periodic images are added twice and others not at
 * all.  or_grid_nc2c_fold(..., fold = 1) restates that loop exactly (a
 * per-cell multiplicity for each periodic image), so the oracle can be
 * pinned to the reference in 3D too; the product and the default oracle keep
 * the periodic fold, which the FP64 direct NDFT adjoint confirms.
 *
 * Kernel weights are computed in float exactly as the reference writes them
 * (host arithmetic, no fused multiply-add except the trajectory scaling, which
 * the reference evaluates on the device where nvcc contracts it).  Sums are
 * accumulated in double, so the oracle is the reference's algorithm with its
 * FP32 summation error removed.
 *
 * Layouts: complex arrays are interleaved (re, im) doubles, x fastest; the
 * batch (coil) axis is outermost, then frames, as in the reference
 * ([grid..., frames, batches] and [samples, frames, batches]).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAXD 4

float or_bessi0f(float x)
{
    float denominator, numerator, z;
    if (x == 0.0f)
        return 1.0f;
    z = x * x;
    numerator = (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z * (z *
                 (z * 0.210580722890567e-22f + 0.380715242345326e-19f) +
                 0.479440257548300e-16f) + 0.435125971262668e-13f) +
                 0.300931127112960e-10f) + 0.160224679395361e-7f) +
                 0.654858370096785e-5f) + 0.202591084143397e-2f) +
                 0.463076284721000e0f) + 0.754337328948189e2f) +
                 0.830792541809429e4f) + 0.571661130563785e6f) +
                 0.216415572361227e8f) + 0.356644482244025e9f) +
                 0.144048298227235e10f);
    denominator = (z * (z * (z - 0.307646912682801e4f) + 0.347626332405882e7f) -
                   0.144048298227235e10f);
    return -numerator / denominator;
}

float or_kb1f(float u, float matrix_size_os, float one_over_W, float beta)
{
    float _tmp = 2.0f * u * one_over_W;
    float tmp = _tmp * _tmp;
    float arg = beta * sqrtf(1.0f - tmp);
    float bessi = or_bessi0f(arg);
    return matrix_size_os * bessi * one_over_W;
}

/* beta per dimension, in float as the reference computes it on the host. */
void or_compute_beta(int D, const uint64_t *N, const uint64_t *mos, float W,
                     float *beta_out)
{
    for (int d = 0; d < D; d++) {
        float os = (float)mos[d] / (float)N[d];
        float w2 = W * W;
        float os2 = os * os;
        float h = os - 0.5f;
        float arg = w2 / os2 * (h * h) - 0.8f;
        beta_out[d] = (float)M_PI * sqrtf(arg);
    }
}

/* ConvolutionKernel::get for the Kaiser kernel: 0 if any |delta_d| > radius,
 * else the product of the per-dimension KB values (left to right). */
float or_kb_get(int D, const float *delta, const float *mos_f, float one_over_W,
                const float *beta, float radius)
{
    for (int d = 0; d < D; d++)
        if (delta[d] > radius)
            return 0.0f;
    float w = or_kb1f(delta[0], mos_f[0], one_over_W, beta[0]);
    for (int d = 1; d < D; d++)
        w = w * or_kb1f(delta[d], mos_f[d], one_over_W, beta[d]);
    return w;
}

/* Per-dimension value of the separable kernel with the radius check,
 * exposed for checks of the CUDA weight tables. */
float or_kb_get_1d(float delta, float mos_f, float one_over_W, float beta,
                   float radius)
{
    if (delta > radius)
        return 0.0f;
    return or_kb1f(delta, mos_f, one_over_W, beta);
}

typedef struct {
    int D;
    int64_t mos[OR_MAXD];
    int64_t pad;           /* 2*ceil(W/2) */
    float mos_f[OR_MAXD];
    float beta[OR_MAXD];
    float W, radius, one_over_W;
} or_plan;

static void or_plan_init(or_plan *p, int D, const uint64_t *N,
                         const uint64_t *mos, float W)
{
    p->D = D;
    p->W = W;
    p->radius = W / 2.0f;
    p->one_over_W = 1.0f / W;
    p->pad = 2 * (int64_t)ceilf(p->radius);
    for (int d = 0; d < D; d++) {
        p->mos[d] = (int64_t)mos[d];
        p->mos_f[d] = (float)mos[d];
    }
    or_compute_beta(D, N, mos, W, p->beta);
}

/* Trajectory in [-1/2,1/2] (float, AoS: D floats per sample) to padded grid
 * units.  Returns 0 on success, 1 if a coordinate is out of range (the
 * reference throws in that case: cuGriddingConvolution.cu:145-152). */
int or_scale_trajectory(int D, const uint64_t *N, const uint64_t *mos, float W,
                        const float *traj, int64_t n, float *scaled)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    for (int64_t i = 0; i < n * D; i++)
        if (!(traj[i] >= -0.5f && traj[i] <= 0.5f))
            return 1;
    for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < D; d++) {
            float bias = (float)((p.mos[d] + p.pad) >> 1);
            scaled[i * D + d] = fmaf(traj[i * D + d], p.mos_f[d], bias);
        }
    return 0;
}

static inline int64_t or_wrap(int64_t x, int64_t m)
{
    x %= m;
    return x < 0 ? x + m : x;
}

/* Multiplicity with which the reference's fold adds the periodic image at
 * stride sigma (each component -1, 0, +1) to a cell whose per-dimension
 * state is st (0 interior, 1 within the ring width of the low face, 2 of the
 * high face): the combination/stride loop of wrap_image_kernel
 * (ConvolverNC2C_standard.cuh:394-437), including its `i & combination`
 * dimension test.  sigma = 0 (the cell itself) always counts once. */
static int or_ref_fold_multiplicity(int D, const int *st, const int *sigma)
{
    int zero = 1;
    for (int d = 0; d < D; d++)
        zero &= sigma[d] == 0;
    if (zero)
        return 1;
    int count = 0;
    for (int comb = 1; comb < (1 << D); comb++) {
        int nd = 0;
        for (int i = 0; i < D; i++)
            nd += (comb & (1 << i)) != 0;
        for (int sel = 0; sel < (1 << nd); sel++) {
            int stride[OR_MAXD], wraps = 0, skipped = 0;
            for (int i = 1; i <= D; i++) {
                stride[i - 1] = 0;
                if (i & comb) {
                    if (i & (sel << skipped)) {
                        if (st[i - 1] == 2) { stride[i - 1] = -1; wraps++; }
                    } else {
                        if (st[i - 1] == 1) { stride[i - 1] = 1; wraps++; }
                    }
                } else {
                    skipped++;
                }
            }
            if (wraps == nd) {
                int same = 1;
                for (int d = 0; d < D; d++)
                    same &= stride[d] == sigma[d];
                count += same;
                break;
            }
        }
    }
    return count;
}

/* Gridding NC2C (the adjoint convolution).  samples: [nb][F][M] complex
 * double; grid_out: [nb][F][prod(mos)] complex double, overwritten (or added
 * to when accumulate != 0).  scaled: [F][M] D-vectors from
 * or_scale_trajectory.  The reference's padded grid and wrap pass are
 * reproduced by folding each padded cell p onto (p - pad/2) mod mos, with
 * multiplicity 1 (fold 0, periodic) or the reference's multiplicity (fold 1,
 * see the header). */
void or_grid_nc2c_fold(int D, const uint64_t *N, const uint64_t *mos, float W,
                       int64_t M, int64_t F, int64_t nb, const float *scaled,
                       const double *samples, double *grid_out, int accumulate, int fold)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    int64_t G = 1;
    for (int d = 0; d < D; d++) G *= p.mos[d];
    const int64_t hw = p.pad / 2;
    const float half_W = 0.5f * W;
    if (!accumulate)
        memset(grid_out, 0, sizeof(double) * 2 * (size_t)(G * F * nb));

#pragma omp parallel for schedule(static)
    for (int64_t bf = 0; bf < nb * F; bf++) {
        const int64_t f = bf % F;
        double *grid = grid_out + 2 * bf * G;
        const double *smp = samples + 2 * bf * M;
        for (int64_t j = 0; j < M; j++) {
            const float *s = scaled + (f * M + j) * D;
            int64_t lo[OR_MAXD], hi[OR_MAXD], cnt[OR_MAXD];
            int64_t ntaps = 1;
            for (int d = 0; d < D; d++) {
                lo[d] = (int64_t)(unsigned int)ceilf(s[d] - half_W);
                hi[d] = (int64_t)(unsigned int)floorf(s[d] + half_W);
                cnt[d] = hi[d] - lo[d] + 1;
                ntaps *= cnt[d];
            }
            const double yr = smp[2 * j], yi = smp[2 * j + 1];
            for (int64_t t = 0; t < ntaps; t++) {
                int64_t rem = t, idx = 0, stride = 1;
                float delta[OR_MAXD];
                int st[OR_MAXD], sigma[OR_MAXD];
                for (int d = 0; d < D; d++) {
                    int64_t pc = lo[d] + rem % cnt[d];
                    rem /= cnt[d];
                    delta[d] = fabsf(s[d] - (float)pc);
                    const int64_t u = pc - hw;                 /* unwrapped cell */
                    const int64_t co = or_wrap(u, p.mos[d]);
                    sigma[d] = u < 0 ? -1 : (u >= p.mos[d] ? 1 : 0);
                    st[d] = co < hw ? 1 : (co >= p.mos[d] - hw ? 2 : 0);
                    idx += co * stride;
                    stride *= p.mos[d];
                }
                float w = or_kb_get(D, delta, p.mos_f, p.one_over_W, p.beta, p.radius);
                if (!isfinite(w))
                    continue;
                double mult = 1.0;
                if (fold == 1)
                    mult = (double)or_ref_fold_multiplicity(D, st, sigma);
                grid[2 * idx] += mult * (double)w * yr;
                grid[2 * idx + 1] += mult * (double)w * yi;
            }
        }
    }
}

void or_grid_nc2c(int D, const uint64_t *N, const uint64_t *mos, float W,
                  int64_t M, int64_t F, int64_t nb, const float *scaled,
                  const double *samples, double *grid_out, int accumulate)
{
    or_grid_nc2c_fold(D, N, mos, W, M, F, nb, scaled, samples, grid_out, accumulate, 0);
}

/* Degridding C2NC (the forward convolution).  grid: [nb][F][prod(mos)]
 * complex double; samples_out: [nb][F][M] complex double, overwritten (or
 * added to when accumulate != 0). */
void or_degrid_c2nc(int D, const uint64_t *N, const uint64_t *mos, float W,
                    int64_t M, int64_t F, int64_t nb, const float *scaled,
                    const double *grid_in, double *samples_out, int accumulate)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    int64_t G = 1;
    for (int d = 0; d < D; d++) G *= p.mos[d];
    const float hw_f = (float)(p.pad >> 1);

#pragma omp parallel for schedule(static)
    for (int64_t bf = 0; bf < nb * F; bf++) {
        const int64_t f = bf % F;
        const double *grid = grid_in + 2 * bf * G;
        double *out = samples_out + 2 * bf * M;
        for (int64_t j = 0; j < M; j++) {
            const float *sp = scaled + (f * M + j) * D;
            float s[OR_MAXD];
            int64_t lo[OR_MAXD], cnt[OR_MAXD];
            int64_t ntaps = 1;
            for (int d = 0; d < D; d++) {
                s[d] = sp[d] - hw_f;
                lo[d] = (int64_t)(int)ceilf(s[d] - p.radius);
                int64_t hi = (int64_t)(int)floorf(s[d] + p.radius);
                cnt[d] = hi - lo[d] + 1;
                if (cnt[d] < 0) cnt[d] = 0;
                ntaps *= cnt[d];
            }
            double ar = 0.0, ai = 0.0;
            for (int64_t t = 0; t < ntaps; t++) {
                int64_t rem = t, idx = 0, stride = 1;
                float delta[OR_MAXD];
                for (int d = 0; d < D; d++) {
                    int64_t g = lo[d] + rem % cnt[d];
                    rem /= cnt[d];
                    delta[d] = fabsf(s[d] - (float)g);
                    idx += or_wrap(g, p.mos[d]) * stride;
                    stride *= p.mos[d];
                }
                float w = or_kb_get(D, delta, p.mos_f, p.one_over_W, p.beta, p.radius);
                if (!isfinite(w))
                    continue;
                ar += (double)w * grid[2 * idx];
                ai += (double)w * grid[2 * idx + 1];
            }
            if (accumulate) {
                out[2 * j] += ar;
                out[2 * j + 1] += ai;
            } else {
                out[2 * j] = ar;
                out[2 * j + 1] = ai;
            }
        }
    }
}

/* The kernel image used for the deapodization filter: one sample at mos/2,
 * evaluated at every cell of the oversampled grid (float values). */
void or_deapod_kernel_image(int D, const uint64_t *N, const uint64_t *mos,
                            float W, float *out)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    int64_t G = 1;
    for (int d = 0; d < D; d++) G *= p.mos[d];
    for (int64_t idx = 0; idx < G; idx++) {
        int64_t rem = idx;
        float delta[OR_MAXD];
        for (int d = 0; d < D; d++) {
            int64_t c = rem % p.mos[d];
            rem /= p.mos[d];
            float sample_pos = 0.5f * p.mos_f[d];
            delta[d] = fabsf(sample_pos - (float)c);
        }
        out[idx] = or_kb_get(D, delta, p.mos_f, p.one_over_W, p.beta, p.radius);
    }
}

/* Direct non-uniform DFT in double precision (the accuracy oracle):
 *   y_j = dcw_j / sqrt(G) * sum_n x_n exp(-2 pi i k_j . (n - N/2))
 * x: [nb][prod(N)] complex, traj: [M] D-vectors (double), y: [nb][M].
 * Separable phases: per sample one table of exp(-2 pi i k_d (n_d - N_d/2))
 * per dimension. */
void or_ndft_forward(int D, const uint64_t *N, double inv_sqrt_G, int64_t M,
                     int64_t nb, const double *traj, const double *dcw,
                     const double *x, double *y)
{
    int64_t NN = 1, maxN = 0;
    for (int d = 0; d < D; d++) {
        NN *= (int64_t)N[d];
        if ((int64_t)N[d] > maxN) maxN = (int64_t)N[d];
    }
#pragma omp parallel
    {
        double *ph = (double *)malloc(sizeof(double) * 2 * (size_t)(D * maxN));
#pragma omp for schedule(dynamic, 16)
        for (int64_t j = 0; j < M; j++) {
            for (int d = 0; d < D; d++)
                for (int64_t n = 0; n < (int64_t)N[d]; n++) {
                    double a = -2.0 * M_PI * traj[j * D + d] *
                               ((double)n - (double)(N[d] / 2));
                    ph[2 * (d * maxN + n)] = cos(a);
                    ph[2 * (d * maxN + n) + 1] = sin(a);
                }
            for (int64_t b = 0; b < nb; b++) {
                const double *xb = x + 2 * b * NN;
                double sr = 0.0, si = 0.0;
                for (int64_t idx = 0; idx < NN; idx++) {
                    int64_t rem = idx;
                    double er = 1.0, ei = 0.0;
                    for (int d = 0; d < D; d++) {
                        int64_t n = rem % (int64_t)N[d];
                        rem /= (int64_t)N[d];
                        double pr = ph[2 * (d * maxN + n)], pi = ph[2 * (d * maxN + n) + 1];
                        double tr = er * pr - ei * pi;
                        ei = er * pi + ei * pr;
                        er = tr;
                    }
                    sr += er * xb[2 * idx] - ei * xb[2 * idx + 1];
                    si += er * xb[2 * idx + 1] + ei * xb[2 * idx];
                }
                double w = dcw ? dcw[j] : 1.0;
                y[2 * (b * M + j)] = sr * inv_sqrt_G * w;
                y[2 * (b * M + j) + 1] = si * inv_sqrt_G * w;
            }
        }
        free(ph);
    }
}

/* Adjoint direct NDFT:
 *   x_n = 1/sqrt(G) * sum_j dcw_j y_j exp(+2 pi i k_j . (n - N/2)). */
void or_ndft_adjoint(int D, const uint64_t *N, double inv_sqrt_G, int64_t M,
                     int64_t nb, const double *traj, const double *dcw,
                     const double *y, double *x)
{
    int64_t NN = 1, maxN = 0;
    for (int d = 0; d < D; d++) {
        NN *= (int64_t)N[d];
        if ((int64_t)N[d] > maxN) maxN = (int64_t)N[d];
    }
    memset(x, 0, sizeof(double) * 2 * (size_t)(NN * nb));
#pragma omp parallel
    {
        double *ph = (double *)malloc(sizeof(double) * 2 * (size_t)(D * maxN));
        double *acc = (double *)calloc(2 * (size_t)(NN * nb), sizeof(double));
#pragma omp for schedule(dynamic, 16)
        for (int64_t j = 0; j < M; j++) {
            for (int d = 0; d < D; d++)
                for (int64_t n = 0; n < (int64_t)N[d]; n++) {
                    double a = 2.0 * M_PI * traj[j * D + d] *
                               ((double)n - (double)(N[d] / 2));
                    ph[2 * (d * maxN + n)] = cos(a);
                    ph[2 * (d * maxN + n) + 1] = sin(a);
                }
            double w = dcw ? dcw[j] : 1.0;
            for (int64_t b = 0; b < nb; b++) {
                double yr = y[2 * (b * M + j)] * w, yi = y[2 * (b * M + j) + 1] * w;
                double *xb = acc + 2 * b * NN;
                for (int64_t idx = 0; idx < NN; idx++) {
                    int64_t rem = idx;
                    double er = 1.0, ei = 0.0;
                    for (int d = 0; d < D; d++) {
                        int64_t n = rem % (int64_t)N[d];
                        rem /= (int64_t)N[d];
                        double pr = ph[2 * (d * maxN + n)], pi = ph[2 * (d * maxN + n) + 1];
                        double tr = er * pr - ei * pi;
                        ei = er * pi + ei * pr;
                        er = tr;
                    }
                    xb[2 * idx] += er * yr - ei * yi;
                    xb[2 * idx + 1] += er * yi + ei * yr;
                }
            }
        }
#pragma omp critical
        for (int64_t i = 0; i < 2 * NN * nb; i++)
            x[i] += acc[i] * inv_sqrt_G;
        free(acc);
        free(ph);
    }
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* d/du of the 1D kernel value for u in [0, radius], derivative of the same
 * rational approximation: phi(u) = mos/W * R(beta^2 (1 - (2u/W)^2)) with
 * R(z) = -num(z)/den(z) the function bessi0 evaluates at z = x^2
 * (ConvolutionKernel.hpp:39-68), so phi'(u) = -(8 mos beta^2 u / W^3) R'(z).
 * Double precision. */
static double or_kb_deriv_1d(double u, double mos_f, double W, double beta, double radius)
{
    static const double a[15] = {0.144048298227235e10, 0.356644482244025e9, 0.216415572361227e8,
                                 0.571661130563785e6,  0.830792541809429e4, 0.754337328948189e2,
                                 0.463076284721000e0,  0.202591084143397e-2, 0.654858370096785e-5,
                                 0.160224679395361e-7, 0.300931127112960e-10, 0.435125971262668e-13,
                                 0.479440257548300e-16, 0.380715242345326e-19, 0.210580722890567e-22};
    if (u > radius)
        return 0.0;
    double t = 2.0 * u / W;
    double z = beta * beta * (1.0 - t * t);
    double num = a[14], dnum = 0.0;
    for (int i = 13; i >= 0; --i) {
        dnum = dnum * z + num;
        num = num * z + a[i];
    }
    const double b2 = -0.307646912682801e4, b1 = 0.347626332405882e7, b0 = -0.144048298227235e10;
    double den = ((z + b2) * z + b1) * z + b0;
    double dden = (3.0 * z + 2.0 * b2) * z + b1;
    double dR = -(dnum * den - num * dden) / (den * den);
    return -8.0 * mos_f * beta * beta * u / (W * W * W) * dR;
}

/* Trajectory gradient of the degridding convolution (oracle for the CUDA
 * gradient kernel): for each sample j and dimension d,
 *   out[j][d] = mos_d * sum_b Re( w[b][j] * sum_taps dphi/ds_d * grid[b][tap] )
 * with the taps, wrap and float kernel values of or_degrid_c2nc.  grid:
 * [nb][F][G] complex double; w: [nb][F][M] complex double; out: [F*M][D]. */
void or_degrid_traj_grad(int D, const uint64_t *N, const uint64_t *mos, float W,
                         int64_t M, int64_t F, int64_t nb, const float *scaled,
                         const double *grid_in, const double *w, double *out)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    int64_t G = 1;
    for (int d = 0; d < D; d++) G *= p.mos[d];
    const float hw_f = (float)(p.pad >> 1);

#pragma omp parallel for schedule(static)
    for (int64_t fj = 0; fj < F * M; fj++) {
        const int64_t f = fj / M, j = fj % M;
        const float *sp = scaled + fj * D;
        float s[OR_MAXD];
        int64_t lo[OR_MAXD], cnt[OR_MAXD];
        int64_t ntaps = 1;
        for (int d = 0; d < D; d++) {
            s[d] = sp[d] - hw_f;
            lo[d] = (int64_t)(int)ceilf(s[d] - p.radius);
            int64_t hi = (int64_t)(int)floorf(s[d] + p.radius);
            cnt[d] = hi - lo[d] + 1;
            if (cnt[d] < 0) cnt[d] = 0;
            ntaps *= cnt[d];
        }
        double acc[OR_MAXD];
        for (int d = 0; d < D; d++) acc[d] = 0.0;
        for (int64_t b = 0; b < nb; b++) {
            const double *grid = grid_in + 2 * (b * F + f) * G;
            const double wr = w[2 * ((b * F + f) * M + j)], wi = w[2 * ((b * F + f) * M + j) + 1];
            for (int64_t t = 0; t < ntaps; t++) {
                int64_t rem = t, idx = 0, stride = 1;
                double val[OR_MAXD], der[OR_MAXD];
                for (int d = 0; d < D; d++) {
                    int64_t g = lo[d] + rem % cnt[d];
                    rem /= cnt[d];
                    double diff = (double)s[d] - (double)g;
                    float delta = fabsf(s[d] - (float)g);
                    val[d] = (double)or_kb_get_1d(delta, p.mos_f[d], p.one_over_W, p.beta[d], p.radius);
                    der[d] = or_kb_deriv_1d(fabs(diff), p.mos_f[d], p.W, p.beta[d], p.radius) * (diff < 0 ? -1.0 : 1.0);
                    idx += or_wrap(g, p.mos[d]) * stride;
                    stride *= p.mos[d];
                }
                const double gr = grid[2 * idx], gi = grid[2 * idx + 1];
                for (int d = 0; d < D; d++) {
                    double c = der[d];
                    for (int e = 0; e < D; e++)
                        if (e != d) c *= val[e];
                    /* Re(w * c * g) */
                    acc[d] += c * (wr * gr - wi * gi);
                }
            }
        }
        for (int d = 0; d < D; d++) out[fj * D + d] = acc[d] * (double)p.mos_f[d];
    }
}

/* ------------------------------------------------------------------------
 * The reference's CPU gridding (hoGriddingConvolution with its
 * ConvolutionMatrix), restated in float for the timed CPU baseline:
 *   - scaling without padding, s = (k + 1/2) * mos:
 *                                   toolboxes/nfft/cpu/hoGriddingConvolution.cpp:50-57
 *   - per sample, the taps i in [ceil(s - W/2), floor(s + W/2)] per
 *     dimension (last dimension outermost, x innermost), wrapped modulo mos,
 *     weight kernel.get(|i - s|):    toolboxes/nfft/cpu/ConvolutionMatrix.cpp:18-76,84-100
 *   - the transpose (per cell, its samples in increasing order):
 *                                   ConvolutionMatrix.cpp:104-137
 *   - C2NC: samples[j] += sum_n grid[idx[n]] * w[n];  NC2C: grid[g] +=
 *     sum_n samples[j_n] * w_n, complext<float> arithmetic, OpenMP over the
 *     batches (coils):              hoGriddingConvolution.cpp:86-150
 * ------------------------------------------------------------------------ */

typedef struct {
    int64_t M, G;
    int64_t *row_ptr;      /* [M+1] per sample */
    uint32_t *row_idx;     /* grid cell of each tap */
    float *row_w;
    int64_t *col_ptr;      /* [G+1] per cell (transpose) */
    uint32_t *col_idx;     /* sample of each tap */
    float *col_w;
} ho_matrix;

void *ho_matrix_create(int D, const uint64_t *N, const uint64_t *mos, float W,
                       const float *traj, int64_t M)
{
    or_plan p;
    or_plan_init(&p, D, N, mos, W);
    ho_matrix *m = (ho_matrix *)calloc(1, sizeof(ho_matrix));
    int64_t G = 1;
    for (int d = 0; d < D; d++) G *= p.mos[d];
    m->M = M;
    m->G = G;
    m->row_ptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(M + 1));
    /* pass 1: taps per sample */
    m->row_ptr[0] = 0;
    for (int64_t j = 0; j < M; j++) {
        int64_t n = 1;
        for (int d = 0; d < D; d++) {
            const float s = (traj[j * D + d] + 0.5f) * p.mos_f[d];
            n *= (int64_t)floorf(s + p.radius) - (int64_t)ceilf(s - p.radius) + 1;
        }
        m->row_ptr[j + 1] = m->row_ptr[j] + n;
    }
    const int64_t nnz = m->row_ptr[M];
    m->row_idx = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nnz);
    m->row_w = (float *)malloc(sizeof(float) * (size_t)nnz);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < M; j++) {
        float s[OR_MAXD];
        int64_t lo[OR_MAXD], cnt[OR_MAXD], stride[OR_MAXD];
        int64_t ntaps = 1, st = 1;
        for (int d = 0; d < D; d++) {
            s[d] = (traj[j * D + d] + 0.5f) * p.mos_f[d];
            lo[d] = (int64_t)ceilf(s[d] - p.radius);
            cnt[d] = (int64_t)floorf(s[d] + p.radius) - lo[d] + 1;
            stride[d] = st;
            st *= p.mos[d];
            ntaps *= cnt[d];
        }
        int64_t o = m->row_ptr[j];
        for (int64_t t = 0; t < ntaps; t++) {
            /* x innermost, the last dimension outermost */
            int64_t rem = t, idx = 0;
            float delta[OR_MAXD];
            for (int d = 0; d < D; d++) {
                const int64_t i = lo[d] + rem % cnt[d];
                rem /= cnt[d];
                delta[d] = fabsf((float)i - s[d]);
                idx += ((i + p.mos[d]) % p.mos[d]) * stride[d];
            }
            m->row_idx[o] = (uint32_t)idx;
            m->row_w[o] = or_kb_get(D, delta, p.mos_f, p.one_over_W, p.beta, p.radius);
            o++;
        }
    }
    /* transpose by counting sort over cells (samples stay in order) */
    m->col_ptr = (int64_t *)calloc((size_t)(G + 1), sizeof(int64_t));
    for (int64_t n = 0; n < nnz; n++) m->col_ptr[m->row_idx[n] + 1]++;
    for (int64_t g = 0; g < G; g++) m->col_ptr[g + 1] += m->col_ptr[g];
    m->col_idx = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nnz);
    m->col_w = (float *)malloc(sizeof(float) * (size_t)nnz);
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)G);
    memcpy(fill, m->col_ptr, sizeof(int64_t) * (size_t)G);
    for (int64_t j = 0; j < M; j++)
        for (int64_t n = m->row_ptr[j]; n < m->row_ptr[j + 1]; n++) {
            const int64_t at = fill[m->row_idx[n]]++;
            m->col_idx[at] = (uint32_t)j;
            m->col_w[at] = m->row_w[n];
        }
    free(fill);
    return m;
}

void ho_matrix_destroy(void *h)
{
    ho_matrix *m = (ho_matrix *)h;
    if (!m) return;
    free(m->row_ptr); free(m->row_idx); free(m->row_w);
    free(m->col_ptr); free(m->col_idx); free(m->col_w);
    free(m);
}

/* grid: [nb][G] complex float; samples: [nb][M] complex float */
void ho_c2nc(void *h, int64_t nb, const float *grid, float *samples, int accumulate)
{
    const ho_matrix *m = (const ho_matrix *)h;
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; b++) {
        const float *g = grid + 2 * b * m->G;
        float *y = samples + 2 * b * m->M;
        for (int64_t j = 0; j < m->M; j++) {
            float re = accumulate ? y[2 * j] : 0.0f, im = accumulate ? y[2 * j + 1] : 0.0f;
            for (int64_t n = m->row_ptr[j]; n < m->row_ptr[j + 1]; n++) {
                const float w = m->row_w[n];
                re += g[2 * (int64_t)m->row_idx[n]] * w;
                im += g[2 * (int64_t)m->row_idx[n] + 1] * w;
            }
            y[2 * j] = re;
            y[2 * j + 1] = im;
        }
    }
}

void ho_nc2c(void *h, int64_t nb, const float *samples, float *grid, int accumulate)
{
    const ho_matrix *m = (const ho_matrix *)h;
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; b++) {
        const float *y = samples + 2 * b * m->M;
        float *g = grid + 2 * b * m->G;
        for (int64_t c = 0; c < m->G; c++) {
            float re = accumulate ? g[2 * c] : 0.0f, im = accumulate ? g[2 * c + 1] : 0.0f;
            for (int64_t n = m->col_ptr[c]; n < m->col_ptr[c + 1]; n++) {
                const float w = m->col_w[n];
                re += y[2 * (int64_t)m->col_idx[n]] * w;
                im += y[2 * (int64_t)m->col_idx[n] + 1] * w;
            }
            g[2 * c] = re;
            g[2 * c + 1] = im;
        }
    }
}
