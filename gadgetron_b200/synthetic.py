"""Seeded synthetic inputs for the non-Cartesian path: trajectories, density
compensation weights, phantoms and coil sensitivity maps.

Conventions follow the reference's own generators where it has them:

* golden-ratio radial profiles: ``toolboxes/core/gpu/radial_utilities.cu:19-45``
  (angle step pi/phi, profile angle (p + offset)*step + pi, sample position
  (i - S/2)/S along the profile, so k lies in [-1/2, 1/2));
* density compensation passed to the SENSE operator as sqrt(w), data
  pre-multiplied by sqrt(w): ``gadgets/pmri/gpuCgSenseGadget.cpp:129,179``.

All generators use ``numpy.random.default_rng(seed)`` and compute in float64,
returning float32 trajectories and complex64 arrays.  Arrays use C order with
x on the last axis; trajectories are [M, D] (or [F, M, D]) with component 0 = x.
"""
from __future__ import annotations

import numpy as np

GOLDEN_ANGLE = np.pi / ((np.sqrt(5.0) + 1.0) * 0.5)


def radial_golden_angle_2d(num_profiles: int, samples_per_profile: int,
                           profile_offset: int = 0) -> np.ndarray:
    """[P*S, 2] float32 golden-ratio radial trajectory."""
    S = samples_per_profile
    p = np.arange(num_profiles, dtype=np.float64) + profile_offset
    ang = p * GOLDEN_ANGLE + np.pi
    r = (np.arange(S, dtype=np.float64) - S * 0.5) / S
    kx = r[None, :] * np.cos(ang)[:, None]
    ky = r[None, :] * np.sin(ang)[:, None]
    return np.stack([kx, ky], axis=-1).reshape(-1, 2).astype(np.float32)


def kooshball_golden_means_3d(num_profiles: int, samples_per_profile: int) -> np.ndarray:
    """[P*S, 3] float32 3D radial ("kooshball") trajectory with directions from
    the 2D golden means (Chan et al., MRM 2009): the two golden means are the
    fractional increments phi1, phi2 of the eigenvector of the Fibonacci-like
    matrix [[0,1,0],[0,0,1],[1,0,1]]; profile p has z = frac(p*phi1) mapped to
    [-1,1] (here cos(polar)), azimuth 2*pi*frac(p*phi2)."""
    A = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 0.0, 1.0]])
    w, v = np.linalg.eig(A)
    k = int(np.argmax(np.real(w)))
    vec = np.real(v[:, k])
    vec = vec / vec[2]
    phi1, phi2 = float(vec[0]), float(vec[1])
    p = np.arange(num_profiles, dtype=np.float64)
    cos_polar = 2.0 * np.mod(p * phi1, 1.0) - 1.0
    az = 2.0 * np.pi * np.mod(p * phi2, 1.0)
    sin_polar = np.sqrt(np.maximum(0.0, 1.0 - cos_polar ** 2))
    d = np.stack([sin_polar * np.cos(az), sin_polar * np.sin(az), cos_polar], -1)
    S = samples_per_profile
    r = (np.arange(S, dtype=np.float64) - S * 0.5) / S
    return (r[None, :, None] * d[:, None, :]).reshape(-1, 3).astype(np.float32)


def spiral_archimedean_2d(num_interleaves: int, samples_per_interleave: int,
                          matrix_size: int, center_density: float = 4.0) -> np.ndarray:
    """[I*S, 2] float32 variable-density Archimedean spiral.

    The sampling density rho(r) falls linearly from ``center_density`` at the
    centre to 1 at the edge (r = 1/2): rho(r) = c - 2 (c - 1) r.  The turns of
    the I interleaves are spaced by dr = 1 / (matrix_size * rho(r)) in total,
    i.e. d(theta)/dr = 2 pi matrix_size rho(r) / I, which integrates to
    theta(r) = 2 pi matrix_size / I * (c r - (c - 1) r^2).  Samples are uniform
    in theta; interleave i is rotated by 2 pi i / I."""
    S = samples_per_interleave
    c = float(center_density)
    R = 0.5
    scale = 2.0 * np.pi * matrix_size / num_interleaves
    theta_max = scale * (c * R - (c - 1.0) * R * R)
    th = theta_max * np.arange(S, dtype=np.float64) / S
    q = th / scale                        # = c r - (c-1) r^2
    if c == 1.0:
        r = q
    else:
        r = (c - np.sqrt(np.maximum(c * c - 4.0 * (c - 1.0) * q, 0.0))) / (2.0 * (c - 1.0))
    out = []
    for i in range(num_interleaves):
        a = th + 2.0 * np.pi * i / num_interleaves
        out.append(np.stack([r * np.cos(a), r * np.sin(a)], -1))
    k = np.concatenate(out, 0)
    return np.clip(k, -0.5, 0.5 - 1e-7).astype(np.float32)


def ramp_dcw(traj: np.ndarray, floor_fraction: float = 0.25) -> np.ndarray:
    """|k| ramp density weights normalised to sum 1, with a floor at the centre
    of floor_fraction * (the smallest nonzero radial step)."""
    traj = np.asarray(traj, np.float64)
    r = np.sqrt(np.sum(traj * traj, axis=-1))
    nz = r[r > 0]
    floor = floor_fraction * (nz.min() if nz.size else 1.0)
    w = np.maximum(r, floor)
    return (w / w.sum()).astype(np.float32)


def gaussian_image(shape, seed: int) -> np.ndarray:
    """i.i.d. N(0,1) real and imaginary parts."""
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def ellipse_phantom(shape, num_ellipses: int, seed: int) -> np.ndarray:
    """Sum of random ellipses (2D) or ellipsoids (3D) with amplitudes U(0,1);
    centres, semi-axes and angles come from the seeded generator."""
    rng = np.random.default_rng(seed)
    D = len(shape)
    grids = np.meshgrid(*[(np.arange(n) - n / 2) / n for n in shape], indexing="ij")
    img = np.zeros(shape, np.float64)
    for _ in range(num_ellipses):
        amp = rng.uniform(0.0, 1.0)
        c = rng.uniform(-0.25, 0.25, D)
        ax = rng.uniform(0.05, 0.3, D)
        if D == 2:
            th = rng.uniform(0, np.pi)
            y, x = grids[0] - c[0], grids[1] - c[1]
            xr = x * np.cos(th) + y * np.sin(th)
            yr = -x * np.sin(th) + y * np.cos(th)
            inside = (xr / ax[1]) ** 2 + (yr / ax[0]) ** 2 <= 1.0
        else:
            inside = np.ones(shape, bool)
            acc = np.zeros(shape)
            for d in range(D):
                acc += ((grids[d] - c[d]) / ax[d]) ** 2
            inside = acc <= 1.0
        img[inside] += amp
    return img.astype(np.complex64)


def gaussian_bump_csm(shape, num_coils: int, sigma: float = 0.4,
                      ring_radius: float = 0.3) -> np.ndarray:
    """[C, *shape] coil maps exp(-|x - mu_c|^2 / (2 sigma^2)) with centres on a
    ring (2D) or a golden-spiral sphere (3D) of radius ring_radius (fractions of
    the field of view), a coil-dependent linear phase, normalised by the
    root-sum-of-squares."""
    D = len(shape)
    grids = np.meshgrid(*[(np.arange(n) - n / 2) / n for n in shape], indexing="ij")
    maps = []
    for c in range(num_coils):
        if D == 2:
            a = 2.0 * np.pi * c / num_coils
            mu = ring_radius * np.array([np.sin(a), np.cos(a)])
        else:
            z = 1.0 - 2.0 * (c + 0.5) / num_coils
            rr = np.sqrt(max(0.0, 1.0 - z * z))
            a = c * np.pi * (3.0 - np.sqrt(5.0))
            mu = ring_radius * np.array([z, rr * np.sin(a), rr * np.cos(a)])
        d2 = sum((grids[d] - mu[d]) ** 2 for d in range(D))
        phase = np.exp(1j * 2.0 * np.pi * 0.5 * sum(mu[d] * grids[d] for d in range(D)))
        maps.append(np.exp(-d2 / (2.0 * sigma * sigma)) * phase)
    maps = np.stack(maps, 0)
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    return (maps / rss[None]).astype(np.complex64)


def uneven_frame_spokes(num_frames: int = 64, base: int = 13, mult: int = 37,
                        mod: int = 77):
    """Spokes per frame for the batched uneven dynamic case: base + (f*mult mod mod)."""
    return [base + (f * mult) % mod for f in range(num_frames)]
