"""Shared case builders for the parity tests (seeded synthetic inputs)."""
from __future__ import annotations

import numpy as np

from gadgetron_b200 import synthetic as S

# Relative L2 bound between the CUDA path (FP32) and the oracle (the
# reference algorithm with float weights and double sums).
PARITY_TOL = 1e-5


def radial_case(N=64, alpha=2.0, W=5.5, spokes=32, samples=128, frames=1, seed=0, batches=1):
    mos = int(round(N * alpha))
    traj = np.concatenate([S.radial_golden_angle_2d(spokes, samples, profile_offset=f * spokes)
                           for f in range(frames)], 0)
    dcw = np.concatenate([S.ramp_dcw(traj[f * spokes * samples:(f + 1) * spokes * samples])
                          for f in range(frames)], 0)
    img = S.gaussian_image((batches, frames, N, N), seed)
    return dict(N=(N, N), mos=(mos, mos), W=W, traj=traj, dcw=dcw, img=img, frames=frames,
                M=spokes * samples, batches=batches)


def kooshball_case(N=64, alpha=1.5, W=4.0, spokes=200, samples=64, seed=0, batches=1):
    mos = int(round(N * alpha))
    if mos % 32 or N % 32:
        # the plan (like the reference, cuGriddingConvolution.cu:71-80) takes
        # only multiples of 32: pick N so that N * alpha is one
        raise ValueError("N = %d, alpha = %g gives an oversampled size %d that is not a multiple of 32"
                         % (N, alpha, mos))
    traj = S.kooshball_golden_means_3d(spokes, samples)
    dcw = S.ramp_dcw(traj)
    img = S.gaussian_image((batches, 1, N, N, N), seed)
    return dict(N=(N, N, N), mos=(mos, mos, mos), W=W, traj=traj, dcw=dcw, img=img, frames=1,
                M=spokes * samples, batches=batches)


def rel_l2(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
