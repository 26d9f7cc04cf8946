"""CPU checks of the oracle itself (no GPU): kernel values, exact adjointness,
agreement with the FP64 direct NDFT, the padded-grid/wrap restatement against
a plain-Python loop over the reference's steps, and the CG restatement."""
import numpy as np
import pytest

from oracle import oracle as O
from gadgetron_b200 import synthetic as S


def test_bessi0_rational_matches_i0():
    from scipy.special import i0
    xs = np.linspace(0.0, 15.0, 301)
    v = np.array([O.bessi0f(x) for x in xs])
    ref = i0(xs)
    assert np.max(np.abs(v - ref) / ref) < 2e-6


def test_beta_formula():
    # beta = pi * sqrt(W^2/alpha^2 (alpha - 1/2)^2 - 0.8)  (Beatty 2005)
    for N, mos, W in [(128, 256, 5.5), (128, 192, 4.0), (512, 640, 4.0), (192, 384, 5.5)]:
        a = mos / N
        b = O.kb_beta([N], [mos], W)[0]
        assert abs(b - np.pi * np.sqrt(W * W / (a * a) * (a - 0.5) ** 2 - 0.8)) < 1e-5 * b


def test_kernel_cutoff_and_peak():
    b = O.kb_beta([64], [128], 5.5)[0]
    assert O.kb_get_1d(2.75001, 128, 5.5, b) == 0.0
    peak = O.kb_get_1d(0.0, 128, 5.5, b)
    assert abs(peak - 128 * O.bessi0f(b) / 5.5) < 1e-3 * peak
    # the reference kernel is I0(0) * mos / W at the edge, not zero
    edge = O.kb_get_1d(2.75, 128, 5.5, b)
    assert edge == pytest.approx(128 / 5.5, rel=1e-5) or edge == 0.0


def _py_grid_padded_wrap(N, mos, W, traj, y):
    """Plain-Python restatement of the reference NC2C steps for one frame and
    one batch: scale (ConvolverNC2C_standard.cuh:25-39), per padded cell
    accumulate over the sample footprint (:41-102, :229-292), then fold the
    padding ring periodically (:358-477)."""
    D = len(N)
    r = np.float32(W) / np.float32(2)
    pad = 2 * int(np.ceil(r))
    hw = pad // 2
    beta = O.kb_beta(N, mos, W)
    padded = np.zeros(tuple(m + pad for m in mos[::-1]), np.complex128)
    for j in range(traj.shape[0]):
        # k*mos + bias rounded once (exact in double, so equal to fmaf)
        s = [np.float32(np.float64(traj[j, d]) * mos[d] + ((mos[d] + pad) >> 1)) for d in range(D)]
        lo = [int(np.ceil(np.float32(s[d] - r))) for d in range(D)]
        hi = [int(np.floor(np.float32(s[d] + r))) for d in range(D)]
        for idx in np.ndindex(*[hi[d] - lo[d] + 1 for d in range(D)]):
            p = [lo[d] + idx[d] for d in range(D)]
            w = None
            for d in range(D):
                delta = abs(np.float32(s[d] - np.float32(p[d])))
                v = np.float32(O.kb_get_1d(delta, mos[d], W, beta[d]))
                w = v if w is None else np.float32(w * v)   # float product, x first
            padded[tuple(p[::-1])] += w * y[j]
    out = np.zeros(tuple(mos[::-1]), np.complex128)
    it = np.ndindex(*padded.shape)
    for p in it:
        g = tuple((p[k] - hw) % mos[::-1][k] for k in range(D))
        out[g] += padded[p]
    return out


def test_grid_restatement_matches_python_loops():
    N, mos, W = (32, 32), (64, 64), 5.5
    rng = np.random.default_rng(0)
    traj = rng.uniform(-0.5, 0.5, (40, 2)).astype(np.float32)
    traj[0] = [-0.5, -0.5]
    traj[1] = [0.4999, 0.0]
    traj[2] = [0.0, 0.0]
    y = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    P = O.OraclePlan(N, mos, W)
    P.preprocess(traj[None])
    g = P.convolve_nc2c(y[None, None]).reshape(64, 64)
    ref = _py_grid_padded_wrap(N, mos, W, traj, y)
    assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_degrid_is_transpose_of_grid():
    N, mos, W = (32, 32), (64, 64), 4.0
    rng = np.random.default_rng(1)
    traj = rng.uniform(-0.5, 0.5, (64, 2)).astype(np.float32)
    P = O.OraclePlan(N, mos, W)
    P.preprocess(traj[None])
    g = rng.standard_normal((1, 1, 64, 64)) + 1j * rng.standard_normal((1, 1, 64, 64))
    y = rng.standard_normal((1, 1, 64)) + 1j * rng.standard_normal((1, 1, 64))
    a = np.vdot(P.convolve_c2nc(g).ravel(), y.ravel())
    b = np.vdot(g.ravel(), P.convolve_nc2c(y).ravel())
    assert abs(a - b) <= 1e-12 * abs(a)


@pytest.mark.parametrize("W,alpha", [(5.5, 2.0), (4.0, 1.5)])
def test_nufft_vs_ndft_2d(W, alpha):
    N = 32
    mos = int(N * alpha)
    mos = ((mos + 31) // 32) * 32
    traj = S.radial_golden_angle_2d(24, 64)
    dcw = S.ramp_dcw(traj)
    x = S.gaussian_image((1, 1, N, N), 2)
    P = O.OraclePlan((N, N), (mos, mos), W)
    P.preprocess(traj[None])
    y = P.forward_c2nc(x)
    yr = O.ndft_forward(x[0], traj, (mos, mos))
    tol = 1e-4 if W == 5.5 else 2e-3
    assert O.rel_l2(y, yr) < tol
    xa = P.backwards_nc2c(y, dcw[None])
    xr = O.ndft_adjoint(yr, traj, (N, N), (mos, mos), dcw)
    assert O.rel_l2(xa, xr) < tol


def test_nufft_vs_ndft_3d():
    N, mos, W = 32, 64, 4.0
    traj = S.kooshball_golden_means_3d(50, 32)
    x = S.gaussian_image((1, 1, N, N, N), 3)
    P = O.OraclePlan((N, N, N), (mos, mos, mos), W)
    P.preprocess(traj[None])
    y = P.forward_c2nc(x)
    yr = O.ndft_forward(x[0], traj, (mos, mos, mos))
    assert O.rel_l2(y, yr) < 2e-3   # KB approximation error at W=4


def test_adjointness_and_real_filter():
    N, mos, W = (32, 32), (64, 64), 5.5
    traj = S.radial_golden_angle_2d(16, 64)
    P = O.OraclePlan(N, mos, W)
    P.preprocess(traj[None])
    rng = np.random.default_rng(3)
    x = rng.standard_normal((1, 1, 32, 32)) + 1j * rng.standard_normal((1, 1, 32, 32))
    z = rng.standard_normal((1, 1, traj.shape[0])) + 1j * rng.standard_normal((1, 1, traj.shape[0]))
    a = np.vdot(P.forward_c2nc(x).ravel(), z.ravel())
    b = np.vdot(x.ravel(), P.backwards_nc2c(z).ravel())
    assert abs(a - b) <= 1e-12 * abs(a)
    f = P.deapodization_filter()
    assert np.max(np.abs(f.imag)) <= 1e-12 * np.max(np.abs(f.real))
    # separable up to the float rounding of the kernel image (the reference
    # grids fl(phi_x * phi_y)), which the small transform values at the grid
    # edge amplify to a few 1e-6
    fr = f.real
    outer = np.outer(fr[:, 32], fr[32, :]) / fr[32, 32]
    assert np.max(np.abs(outer - fr) / np.abs(fr)) <= 1e-5


def test_trajectory_range_rejected():
    P = O.OraclePlan((32, 32), (64, 64), 5.5)
    with pytest.raises(ValueError):
        P.preprocess(np.full((1, 8, 2), 0.51, np.float32))


def test_cg_oracle_converges():
    N, mos, W = (32, 32), (64, 64), 5.5
    traj = S.radial_golden_angle_2d(48, 64)
    dcw = S.ramp_dcw(traj)
    csm = S.gaussian_bump_csm((32, 32), 4)
    ph = S.ellipse_phantom((32, 32), 10, 0)[None]
    P = O.OraclePlan(N, mos, W)
    P.preprocess(traj[None])
    E = O.OracleSense(P, csm, np.sqrt(dcw)[None])
    d = E.mult_M(ph)
    hist = []
    x = O.cg_solve(E, d, iterations=20, tc_tolerance=0.0, history=hist)
    assert hist[-1] < hist[0] * 1e-2
    assert O.rel_l2(E.mult_M(x), d) < 0.05


def test_oracle_traj_grad_matches_finite_differences():
    """The oracle's analytic trajectory derivative (derivative of the same
    rational Kaiser-Bessel approximation) against central differences of the
    oracle forward, away from the points where a tap enters the support."""
    N, mos, W = (32, 32), (64, 64), 5.5
    traj = (S.radial_golden_angle_2d(24, 64).astype(np.float64) * 0.999).astype(np.float32)
    M = traj.shape[0]
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 1, 32, 32)) + 1j * rng.standard_normal((2, 1, 32, 32))
    v = rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))
    P = O.OraclePlan(N, mos, W)
    P.preprocess(traj[None])
    g = P.traj_grad_forward(x, np.conj(v))
    h = 1e-4
    fd = np.zeros((M, 2))
    for d in range(2):
        vals = []
        for sg in (1, -1):
            tp = traj.copy()
            tp[:, d] = (tp[:, d].astype(np.float64) + sg * h).astype(np.float32)
            P2 = O.OraclePlan(N, mos, W)
            P2.preprocess(tp[None])
            y = P2.forward_c2nc(x).reshape(2, M)
            vals.append((np.conj(v) * y).real.sum(0))
        dk = ((traj[:, d].astype(np.float64) + h).astype(np.float32).astype(np.float64) -
              (traj[:, d].astype(np.float64) - h).astype(np.float32).astype(np.float64))
        fd[:, d] = (vals[0] - vals[1]) / dk
    ok = np.ones(M, bool)
    r = W / 2
    for d in range(2):
        lo = (traj[:, d].astype(np.float64) - h) * mos[d] + mos[d] / 2
        hi = (traj[:, d].astype(np.float64) + h) * mos[d] + mos[d] / 2
        for sgn in (-1.0, 1.0):
            ok &= np.ceil(lo + sgn * r - 1e-3) == np.ceil(hi + sgn * r + 1e-3)
            ok &= np.floor(lo + sgn * r - 1e-3) == np.floor(hi + sgn * r + 1e-3)
    idx = np.nonzero(ok)[0]
    assert len(idx) > 0.5 * M
    assert np.linalg.norm(g[idx] - fd[idx]) / np.linalg.norm(fd[idx]) < 1e-3


def test_image_operator_known_answer():
    """imageOperator::compute + cuImageOperator::estimate_offset on a case
    worked by hand: 99 elements 4 and one element 1 (asum 397)."""
    z = np.full(100, 4.0, np.complex64)
    z[37] = 1.0
    img, off = O.image_operator_compute(z)
    scale = np.float32(np.float32(100) / np.float32(397.0))
    a4, a1 = np.float32(np.float32(4.0) * scale), scale
    # a1 / a4 = 0.25 exactly: bin 12500 of 50000; 1% of 100 elements = 1, so
    # the cumulative count first reaches 1 after bin 12500: counter = 12501
    exp_off = np.float32(np.float32(12502) * a4 / np.float32(50000))
    assert off == float(exp_off)
    assert img[0] == np.float32(np.float32(1) / np.float32(a4 + exp_off))
    assert img[37] == np.float32(np.float32(1) / np.float32(a1 + exp_off))
    img2, off2 = O.image_operator_compute(z, offset_estimation=False)
    assert off2 == 0.0
    assert img2[0] == np.float32(np.float32(1) / a4) and img2[37] == np.float32(np.float32(1) / a1)


def test_sense_precond_weights_formula():
    """gpuCgSenseGadget.cpp:167-176: 1 / sqrt(sum_c |csm_c|^2 + kappa R)."""
    csm = np.array([[[3.0, 0.0]], [[4.0j, 1.0]]], np.complex64)   # 2 coils, 1 x 2 pixels
    R = np.array([[2.0, 5.0]], np.float32)
    w = O.sense_precond_weights(csm, R, kappa=0.5)
    np.testing.assert_allclose(w, 1.0 / np.sqrt(np.array([[9 + 16 + 1.0, 0 + 1 + 2.5]])), rtol=1e-12)


def test_cg_regularization_term_is_kappa_R_squared():
    """cgSolver::mult_MH_M with an image regulariser: E^H E x + kappa R^2 x."""
    class Eye:
        def mult_MH(self, y):
            return y

        def mult_MH_M(self, x):
            return x
    d = np.array([1.0 + 1.0j, 2.0, -1.0j])
    R = np.array([1.0, 2.0, 3.0])
    x = O.cg_solve(Eye(), d, iterations=5, tc_tolerance=0.0, regularization=[(0.5, R)])
    np.testing.assert_allclose(x, d / (1.0 + 0.5 * R * R), rtol=1e-12)


def test_radial_trajectory_conventions():
    """The golden-ratio trajectory of radial_utilities.cu:25-44 is the one the
    synthetic workloads use (FP64 there, float32 here); fixed angles cover a
    half turn."""
    t = O.radial_trajectory_golden_ratio_2d(256, 64)
    np.testing.assert_allclose(t.reshape(-1, 2), S.radial_golden_angle_2d(64, 256), atol=1e-5)
    f = O.radial_trajectory_fixed_angle_2d(64, 8, 2)
    ang = np.arctan2(f[0, 0::64, 1], f[0, 0::64, 0])     # first sample of every profile of frame 0
    steps = np.diff(np.unwrap(ang))
    np.testing.assert_allclose(steps, np.pi / 8, atol=1e-5)
    f1 = np.arctan2(f[1, 0, 1], f[1, 0, 0])               # frame 1 is shifted by pi / (8 * 2)
    assert abs(np.angle(np.exp(1j * (f1 - ang[0]))) - np.pi / 16) < 1e-5


def test_radial_dcw_geometry():
    """Voronoi weights (radial_utilities.cu:200-396): with equally spaced
    profiles they are the same on every profile, symmetric about the centre,
    grow linearly away from it, and tile the disc they cover."""
    P, Sn = 64, 128
    w = O.radial_dcw_2d(Sn, P, 1.0, 1.0, golden=False).reshape(P, Sn)
    np.testing.assert_allclose(w, np.broadcast_to(w[:1], w.shape), rtol=1e-4)
    np.testing.assert_allclose(w[0, 1:Sn // 2], w[0, Sn - 1:Sn // 2:-1], rtol=1e-4)
    # ring of radius r at unit radial spacing: 2 pi r / (2 P) per sample
    r = np.abs(np.arange(Sn) - Sn // 2)[Sn // 2 + 1:Sn - 1]
    np.testing.assert_allclose(w[0, Sn // 2 + 1:Sn - 1], np.pi * r / P, rtol=2e-3)
    assert abs(w[0, Sn // 2] - np.pi * 0.25 / P) < 1e-7
    total = w.sum()
    assert abs(total - np.pi * (Sn / 2) ** 2) / (np.pi * (Sn / 2) ** 2) < 0.02


def _sdc_python_loops(traj, N, os_factor, iters, kw):
    """estimate_dcw written out with explicit loops (small cases only)."""
    import math
    R = float(np.float32(0.96960938) * np.float32(kw))
    pad = 2 * math.ceil(R)
    mos = [((int(np.float32(n) * np.float32(os_factor)) + 31) // 32) * 32 for n in N]
    D = len(N)
    pos = []
    for k in traj:
        pos.append([float(np.float32(np.float64(k[d]) * mos[d] + ((mos[d] + pad) >> 1)) - np.float32(pad // 2))
                    for d in range(D)])

    def taps(s):
        rng = [range(math.ceil(s[d] - R), math.floor(s[d] + R) + 1) for d in range(D)]
        out = []
        for cy in (rng[1] if D > 1 else [0]):
            for cx in rng[0]:
                c = [cx, cy][:D]
                ad = [abs(s[d] - c[d]) for d in range(D)]
                w = float(O.jinc_weight(np.array(ad, np.float32), R))
                idx = 0
                for d in range(D - 1, -1, -1):
                    idx = idx * mos[d] + (c[d] % mos[d])
                out.append((idx, w))
        return out
    T = [taps(s) for s in pos]
    w = [1.0] * len(traj)
    for _ in range(iters):
        grid = {}
        for j, tj in enumerate(T):
            for idx, wt in tj:
                grid[idx] = grid.get(idx, 0.0) + wt * w[j]
        t = [sum(wt * grid.get(idx, 0.0) for idx, wt in tj) for tj in T]
        w = [0.0 if t[j] == 0 else w[j] / t[j] for j in range(len(w))]
    return np.array(w)


def test_sdc_restatement_matches_python_loops():
    rng = np.random.default_rng(3)
    traj = rng.uniform(-0.5, 0.5, (40, 2)).astype(np.float32)
    traj[0] = 0.0                      # a sample on a cell centre
    traj[1] = [0.4999, -0.5]           # samples at the wrap
    ref = _sdc_python_loops(traj, (32, 32), 2.0, 3, 4.0)
    np.testing.assert_allclose(O.estimate_dcw(traj, (32, 32), 2.0, 3, 4.0), ref, rtol=1e-12)


def test_sdc_converges_towards_fixed_point():
    """The estimate drives C2NC(NC2C(w)) towards 1 (SDC.hpp:62-77)."""
    traj = S.radial_golden_angle_2d(32, 128).astype(np.float32)
    r0 = O.sdc_fixed_point_residual(traj, (64, 64), 2.0, 5.5, np.ones(traj.shape[0]))
    r10 = O.sdc_fixed_point_residual(traj, (64, 64), 2.0, 5.5, O.estimate_dcw(traj, (64, 64), 2.0, 10, 5.5))
    r30 = O.sdc_fixed_point_residual(traj, (64, 64), 2.0, 5.5, O.estimate_dcw(traj, (64, 64), 2.0, 30, 5.5))
    assert r0 > 10 and r10 < 0.1 and r30 < r10
    # radial density: the estimate grows with |k| away from the centre
    w = O.estimate_dcw(traj, (64, 64), 2.0, 10, 5.5).reshape(32, 128)
    assert w[:, 64 + 40].mean() > 5 * w[:, 64 + 4].mean()


def test_jinc_weight_shape():
    R = np.float32(0.96960938) * np.float32(5.5)
    assert abs(O.jinc_weight(np.zeros((1, 2), np.float32), R)[0] - 0.999923599661866) < 1e-6
    assert O.jinc_weight(np.array([[R * 0.97, 0.0]], np.float32), R)[0] == 0.0    # r >= 0.9696 -> 0
    assert O.jinc_weight(np.array([[R + 0.1, 0.0]], np.float32), R)[0] == 0.0


def test_sense_buffer_running_sum_is_last_cycles():
    """cuBuffer (cuBuffer.cpp:63-134): after each completed slot the running
    sum is the gridded data of exactly the last num_cycles slots."""
    N, mos, W, C = (32, 32), (64, 64), 5.5, 2
    buf = O.OracleSenseBuffer(N, mos, W, C, num_cycles=2, num_sub_cycles=2)
    rng = np.random.default_rng(9)
    frames = []
    for f in range(7):
        t = S.radial_golden_angle_2d(8, 64, profile_offset=8 * f).astype(np.float32)
        y = rng.standard_normal((C, t.shape[0])) + 1j * rng.standard_normal((C, t.shape[0]))
        frames.append((t, y))
    assert np.all(buf.get_accumulated_coil_images() == 1)

    def gridded(fs):
        out = np.zeros((C, 1) + mos[::-1], np.complex128)
        for t, y in fs:
            P = O.OraclePlan(N, mos, W)
            P.preprocess(t.reshape(1, -1, 2))
            out = P.convolve_nc2c(y.reshape(C, 1, -1), accumulate_into=out)
        return out
    done = [buf.add_frame_data(y, t) for t, y in frames]
    assert done == [False, True, False, True, False, True, False]
    np.testing.assert_allclose(buf.acc, gridded(frames[2:6]), rtol=1e-12, atol=1e-12)


def test_b1_map_recovers_uniform_sensitivities():
    """estimate_b1_map (b1_map.cu:29-118): with spatially constant coil
    sensitivities s the correlation matrices are rank one and the estimate is
    s / |s| with coil 0 made real, at every pixel."""
    rng = np.random.default_rng(4)
    s = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    rho = 1.0 + rng.uniform(0, 1, (20, 24))
    imgs = s[:, None, None] * rho[None]
    est = O.estimate_b1_map(imgs, 2)
    exp = s / np.linalg.norm(s) * np.exp(-1j * np.angle(s[0]))
    np.testing.assert_allclose(est, np.broadcast_to(exp[:, None, None], est.shape), atol=1e-12)
    np.testing.assert_allclose(O.estimate_b1_map(imgs, 2, target_coils=3)[:, 5, 5],
                               s[:3] / np.linalg.norm(s[:3]) * np.exp(-1j * np.angle(s[0])), atol=1e-12)


def test_b1_map_box_smoothing_zero_padded():
    """The 7-box of the smoothing counts cells outside the image as zero."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 9, 11)) + 1j * rng.standard_normal((2, 9, 11))
    xn = x / np.sqrt(np.sum(np.abs(x) ** 2, axis=0))[None]
    a01 = xn[1] * np.conj(xn[0])
    ref = np.zeros_like(a01)
    for y in range(9):
        for xx in range(11):
            ref[y, xx] = a01[max(0, y - 3):y + 4, max(0, xx - 3):xx + 4].sum() / 49.0
    # one power iteration from b = 1 with two coils: t_1 = A[0][1] + A[1][1]
    A00 = np.abs(xn[0]) ** 2
    A11 = np.abs(xn[1]) ** 2

    def box(a):
        out = np.zeros_like(a)
        for y in range(9):
            for xx in range(11):
                out[y, xx] = a[max(0, y - 3):y + 4, max(0, xx - 3):xx + 4].sum() / 49.0
        return out
    S00, S11, S01 = box(A00), box(A11), ref
    # A[k][j]: A[0][1] = x_1 conj(x_0) = S01, A[1][0] = conj(S01)
    b = np.ones((2, 9, 11), complex)
    for _ in range(2):
        t0 = S00 * b[0] + np.conj(S01) * b[1]
        t1 = S01 * b[0] + S11 * b[1]
        nrm = np.sqrt(np.abs(t0) ** 2 + np.abs(t1) ** 2)
        b = np.stack([t0 / nrm, t1 / nrm])
    b = b * np.exp(-1j * np.angle(b[0]))[None]
    np.testing.assert_allclose(O.estimate_b1_map(x, 2), b, atol=1e-12)
