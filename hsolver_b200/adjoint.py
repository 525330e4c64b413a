"""Differentiable conjugate-heat-transfer objective over the C ABI.

`ChtProblem` wraps hs_cht_*: with the flow frozen at a Solver's current
velocities it solves the monolithic fluid+solid energy equation for given
solid conductivities (one per solid region) and volumetric sources (one per
cell, used in solid cells) and returns J = (sum_solid T^8 dV)^(1/8).
`ChtObjective` is the torch.autograd.Function around it: its backward is the
hand-written adjoint (one transposed solve), not autograd through the solver.
"""
import ctypes

import numpy as np

from . import HsError, load


class ChtParams(ctypes.Structure):
    _fields_ = [("k_fluid", ctypes.c_double), ("t_boundary", ctypes.c_double), ("tol", ctypes.c_double),
                ("maxiter", ctypes.c_int), ("reserved", ctypes.c_int * 5)]


def _bind(L):
    if getattr(L, "_cht_bound", False):
        return
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.hs_cht_params_default.argtypes = [ctypes.POINTER(ChtParams)]
    L.hs_cht_params_default.restype = None
    L.hs_cht_create.argtypes = [vp, ctypes.POINTER(ChtParams), ctypes.POINTER(vp)]
    L.hs_cht_set_solid.argtypes = [vp, dp, dp]
    L.hs_cht_forward.argtypes = [vp, dp, dp, ip, dp]
    L.hs_cht_adjoint.argtypes = [vp, dp, dp, ip, dp]
    L.hs_cht_velocities.argtypes = [vp, dp, dp, dp]
    L.hs_cht_destroy.argtypes = [vp]
    L.hs_cht_destroy.restype = None
    L._cht_bound = True


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class ChtProblem:
    """Energy solve + adjoint on one Solver's case and current flow."""

    def __init__(self, solver, k_fluid=1.0, t_boundary=293.0, tol=1e-12, maxiter=20000):
        L = load()
        _bind(L)
        self._L = L
        self.solver = solver
        prm = ChtParams()
        L.hs_cht_params_default(ctypes.byref(prm))
        prm.k_fluid, prm.t_boundary, prm.tol, prm.maxiter = k_fluid, t_boundary, tol, maxiter
        h = ctypes.c_void_p()
        rc = L.hs_cht_create(solver.h, ctypes.byref(prm), ctypes.byref(h))
        if rc != 0:
            raise HsError(rc, L.hs_last_error(solver.h).decode())
        self.h = h
        self.N = solver.dims[0] * solver.dims[1] * solver.dims[2]
        self.nreg = solver.nsolid
        self.last = {}

    def __del__(self):
        if getattr(self, "h", None):
            self._L.hs_cht_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise HsError(rc, self._L.hs_last_error(self.solver.h).decode())

    def forward(self, k_region, q_cell, want_T=False):
        k = np.ascontiguousarray(k_region, np.float64)
        q = np.ascontiguousarray(q_cell, np.float64)
        assert k.size == self.nreg and q.size == self.N
        self._check(self._L.hs_cht_set_solid(self.h, _p(k), _p(q)))
        T = np.empty(self.N) if want_T else None
        J, rr, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self._L.hs_cht_forward(self.h, _p(T) if want_T else None, ctypes.byref(J), ctypes.byref(it),
                                           ctypes.byref(rr)))
        self.last = {"forward_iters": it.value, "forward_relres": rr.value}
        return (J.value, T) if want_T else J.value

    def gradient(self):
        """dJ/dq (per cell) and dJ/dk (per solid region) at the last forward."""
        dq = np.empty(self.N)
        dk = np.empty(max(self.nreg, 1))
        rr, it = ctypes.c_double(), ctypes.c_int()
        self._check(self._L.hs_cht_adjoint(self.h, _p(dq), _p(dk), ctypes.byref(it), ctypes.byref(rr)))
        self.last.update({"adjoint_iters": it.value, "adjoint_relres": rr.value})
        return dq, dk[:self.nreg]

    def velocities(self):
        nx, ny, nz = self.solver.dims
        ug, vg, wg = np.empty((nx + 1) * ny * nz), np.empty(nx * (ny + 1) * nz), np.empty(nx * ny * (nz + 1))
        self._check(self._L.hs_cht_velocities(self.h, _p(ug), _p(vg), _p(wg)))
        return ug, vg, wg


def objective_function():
    """torch.autograd.Function for J(q, k); imported lazily so the package
    does not need torch."""
    import torch

    class ChtObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, q, k, problem):
            J = problem.forward(k.detach().cpu().numpy(), q.detach().cpu().numpy())
            ctx.problem = problem
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            dq, dk = ctx.problem.gradient()
            return (gJ * torch.from_numpy(dq), gJ * torch.from_numpy(dk), None)

    return ChtObjective
