"""hs_pcg_solve (the standalone counterpart of the reference's HYPRE PCG call)
against the oracle's CG on a masked, variable-coefficient 7-point system."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_system(nx, ny, nz, seed, symmetric=False):
    """Masked 7-point system; with per-cell random coefficients the matrix is
    non-symmetric like the reference's (each row uses its own cell's
    coefficient for both neighbours), with constant ones it is SPD."""
    rng = np.random.default_rng(seed)
    shape = (nz + 2, ny + 2, nx + 2)
    unknown = np.zeros(shape, bool)
    unknown[1:-1, 1:-1, 1:-1] = True
    # a solid block of non-unknowns and a ragged corner
    unknown[2:5, 3:6, 2:7] = False
    unknown[-2, -2, 1:4] = False
    if symmetric:
        coef = [np.where(unknown, c, 0.0) for c in (1.0, 2.0, 0.5)]
    else:
        coef = [np.where(unknown, rng.uniform(0.5, 2.0, shape), 0.0) for _ in range(3)]
    b = np.where(unknown, rng.standard_normal(shape), 0.0)
    return [c.ravel() for c in coef], b.ravel()


def gpu_solve(nx, ny, nz, coef, b, tol, maxiter):
    import torch
    import hsolver_b200
    L = hsolver_b200.load()
    L.hs_pcg_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_void_p)]
    L.hs_pcg_solve.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_int,
                                                                            ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                                            ctypes.POINTER(ctypes.c_double)]
    L.hs_pcg_destroy.argtypes = [ctypes.c_void_p]
    h = ctypes.c_void_p()
    assert L.hs_pcg_create(nx, ny, nz, 0, ctypes.byref(h)) == 0, L.hs_last_error(None)
    dev = [torch.tensor(a, device="cuda") for a in coef + [b]]
    x = torch.full_like(dev[3], 7.0)
    it, rr = ctypes.c_int(), ctypes.c_double()
    rc = L.hs_pcg_solve(h, *[ctypes.c_void_p(t.data_ptr()) for t in dev], ctypes.c_void_p(x.data_ptr()), tol, maxiter,
                        None, ctypes.byref(it), ctypes.byref(rr))
    L.hs_pcg_destroy(h)
    assert rc == 0
    return x.cpu().numpy(), it.value, rr.value


@pytest.mark.parametrize("dims,seed", [((20, 12, 10), 1), ((33, 17, 9), 2), ((64, 40, 30), 3)])
def test_pcg_matches_oracle(dims, seed):
    from oracle import oracle
    nx, ny, nz = dims
    coef, b = make_system(nx, ny, nz, seed)
    xg, ig, rg = gpu_solve(nx, ny, nz, coef, b, 1e-10, 2000)
    xo, io, ro = oracle.pcg_solve(nx, ny, nz, *coef, b, tol=1e-10, maxiter=2000)
    assert abs(ig - io) <= 1
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-9
    assert abs(rg - ro) <= 1e-6 * max(ro, 1e-30) + 1e-14
    # zero off the unknowns
    assert not np.any(xg[b == 0])


@pytest.mark.parametrize("dims", [(20, 12, 10), (64, 40, 30)])
def test_pcg_converges_on_spd_system(dims):
    from oracle import oracle
    nx, ny, nz = dims
    coef, b = make_system(nx, ny, nz, 5, symmetric=True)
    xg, ig, rg = gpu_solve(nx, ny, nz, coef, b, 1e-10, 2000)
    xo, io, ro = oracle.pcg_solve(nx, ny, nz, *coef, b, tol=1e-10, maxiter=2000)
    assert rg < 1e-10 and ro < 1e-10 and ig < 2000
    assert abs(ig - io) <= 1
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-9


def test_pcg_zero_rhs_and_maxiter():
    nx, ny, nz = 12, 10, 8
    coef, b = make_system(nx, ny, nz, 4)
    x, it, rr = gpu_solve(nx, ny, nz, coef, np.zeros_like(b), 1e-5, 100)
    assert it == 0 and not np.any(x)
    x, it, rr = gpu_solve(nx, ny, nz, coef, b, 1e-30, 7)
    assert it == 7
