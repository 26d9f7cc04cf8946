"""Python mirror of ``cuCgSolver<float_complext>`` (toolboxes/solvers/gpu/cuCgSolver.h,
toolboxes/solvers/cgSolver.h:33-411) over the C ABI.

Defaults follow cgSolver's constructor (cgSolver.h:49-54): 10 iterations,
tc_tolerance 1e-3 with the relative-residual stop rule (rq/rq0 < tol).
Dot products and norms are FP64 on the device; no host synchronisation
happens inside the solve.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream
from .sense import cuNonCartesianSenseOperator


class cuCgSolver:
    def __init__(self):
        h = ctypes.c_void_p()
        check(lib.gb_cg_create(ctypes.byref(h)))
        self._h = h
        self.E = None
        self.iterations = 10
        self.tc_tolerance = 1e-3
        self.x0 = None
        self.precond = None
        self._precond_src = None
        self.reg_ops = []
        self._reg_image = None
        self.refinements = 1
        self.last_iterations = 0
        self.residual_history = None

    def __del__(self):
        if getattr(self, "_h", None) is not None and lib is not None:
            lib.gb_cg_destroy(self._h)
            self._h = None

    def set_encoding_operator(self, op: cuNonCartesianSenseOperator):
        self.E = op
        check(lib.gb_cg_set_encoding_operator(self._h, op._h, ctypes.c_float(op.get_weight())))

    def set_max_iterations(self, iterations: int):
        self.iterations = int(iterations)
        check(lib.gb_cg_set_max_iterations(self._h, self.iterations))

    def get_max_iterations(self) -> int:
        return self.iterations

    def set_tc_tolerance(self, tol: float):
        self.tc_tolerance = float(tol)
        check(lib.gb_cg_set_tc_tolerance(self._h, ctypes.c_float(tol)))

    def get_tc_tolerance(self) -> float:
        return self.tc_tolerance

    def set_x0(self, x0: Optional[torch.Tensor]):
        if x0 is not None:
            _check_tensor(x0, torch.complex64, "x0")
        self.x0 = x0
        check(lib.gb_cg_set_x0(self._h, _ptr(x0)))

    def _frames_of(self, w: torch.Tensor) -> torch.Tensor:
        """Diagonal weights over the solution [frames, N...]: weights of one
        frame are repeated over the frames (the reference broadcasts them)."""
        E = self.E
        n = 1
        for v in E.matrix_size:
            n *= int(v)
        F = max(1, int(E.num_frames))
        if w.numel() == n * F:
            return w.contiguous()
        if w.numel() == n:
            return w.reshape(1, n).repeat(F, 1).contiguous()
        raise ValueError("diagonal weights must hold N... or N... x frames elements")

    def set_preconditioner(self, weights):
        """cgSolver::set_preconditioner: a cuCgPreconditioner, or its real
        diagonal weights directly (applied twice per iteration, as the
        reference does); None clears."""
        if weights is not None and hasattr(weights, "get_weights"):
            weights = weights.get_weights()
        if weights is not None:
            _check_tensor(weights, torch.float32, "weights")
            if self.E is None:
                raise RuntimeError("set_encoding_operator before set_preconditioner")
            weights = self._frames_of(weights)
        self.precond = weights
        check(lib.gb_cg_set_preconditioner(self._h, _ptr(weights)))

    def set_identity_regularization(self, kappa: float):
        check(lib.gb_cg_set_identity_regularization(self._h, ctypes.c_float(kappa)))

    def add_regularization_operator(self, R):
        """cgSolver::add_regularization_operator (linearOperatorSolver.h:38-41)
        for a cuImageOperator: adds R.get_weight() * R^H R to E^H E.  One
        regularisation operator per solver."""
        if self.reg_ops:
            raise RuntimeError("one regularisation operator per solver is supported")
        if self.E is None:
            raise RuntimeError("set_encoding_operator before add_regularization_operator")
        img = self._frames_of(R.get())
        self.reg_ops.append(R)
        self._reg_image = img
        check(lib.gb_cg_set_image_regularization(self._h, _ptr(img), ctypes.c_float(R.get_weight())))

    def clear_regularization_operators(self):
        self.reg_ops = []
        self._reg_image = None
        check(lib.gb_cg_set_identity_regularization(self._h, ctypes.c_float(0.0)))

    def set_refinements(self, n: int):
        self.refinements = int(n)
        check(lib.gb_cg_set_refinements(self._h, self.refinements))

    def set_barrier_spin_limit(self, polls: int):
        """Diagnostic: polls of the fused iteration's grid barrier before a
        block gives up and flags bit 1 of the device error word (0: default)."""
        check(lib.gb_cg_set_barrier_spin_limit(self._h, int(polls)))

    def set_row_fusion(self, enable: bool):
        """2D: x passes of the FFTs fused into the pad and the crop (default)
        or, when disabled, the barrier-synchronised fused tail."""
        check(lib.gb_cg_set_row_fusion(self._h, int(bool(enable))))

    def set_use_graph(self, use: bool):
        check(lib.gb_cg_set_use_graph(self._h, int(bool(use))))

    def set_frame_independent(self, independent: bool):
        """Per-frame CG scalars: each frame of a multi-frame operator is solved
        as its own problem, all frames still in one launch per kernel."""
        check(lib.gb_cg_set_frame_independent(self._h, int(bool(independent))))

    def solve(self, d: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if self.E is None:
            raise RuntimeError("Error: cgSolver::compute_rhs : no encoding operator is set")
        _check_tensor(d, torch.complex64, "d")
        E = self.E
        shape = (E.num_frames,) + tuple(reversed(E.matrix_size))
        if out is None:
            out = torch.empty(shape, dtype=torch.complex64, device=d.device)
        n_hist = max(1, self.iterations * self.refinements)
        if self.residual_history is None or self.residual_history.numel() < n_hist:
            self.residual_history = torch.zeros(n_hist, dtype=torch.float64, device=d.device)
        its = ctypes.c_uint32()
        check(lib.gb_cg_solve(self._h, _ptr(d), _ptr(out), _ptr(self.residual_history), ctypes.byref(its),
                              _stream()))
        self.last_iterations = its.value
        return out
