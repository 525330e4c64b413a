"""hs_pcg_solve_noalloc: the pressure-correction solve for callers that cannot
allocate device memory while they run (their GPU memory belongs to their own
arena, or cudaMalloc/cudaFree would synchronise the device in the middle of
their loop).  It must give the same answer as the allocating hs_pcg_solve and
as the oracle's CG, call after call, although every call reuses one static
scratch array, and it must leave the device's free memory unchanged.

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(nx, ny, nz, seed, symmetric=False):
    """A masked 7-point system: per-cell random coefficients (each row uses
    its own cell's for both neighbours, a non-symmetric matrix like the
    reference's, on which CG runs to its iteration limit), or per-axis
    constants (symmetric positive definite: CG converges)."""
    rng = np.random.default_rng(seed)
    shape = (nz + 2, ny + 2, nx + 2)
    unknown = np.zeros(shape, bool)
    unknown[1:-1, 1:-1, 1:-1] = True
    unknown[2:4, 2:5, 3:7] = False  # a block of non-unknowns
    if symmetric:
        coef = [np.where(unknown, c, 0.0).ravel() for c in (1.0, 2.0, 0.5)]
    else:
        coef = [np.where(unknown, rng.uniform(0.5, 2.0, shape), 0.0).ravel() for _ in range(3)]
    b = np.where(unknown, rng.standard_normal(shape), 0.0).ravel()
    return coef, b


def _lib():
    import hsolver_b200
    L = hsolver_b200.load()
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.hs_pcg_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(vp)]
    L.hs_pcg_solve.argtypes = [vp] + [vp] * 5 + [ctypes.c_double, ctypes.c_int, vp, ip, dp]
    L.hs_pcg_destroy.argtypes = [vp]
    L.hs_pcg_solve_noalloc.argtypes = [ctypes.c_int] * 3 + [vp] * 5 + [ctypes.c_double, ctypes.c_int, vp, ip, dp]
    L.hs_last_error.argtypes = [vp]
    L.hs_last_error.restype = ctypes.c_char_p
    return L


def _ptrs(ts):
    return [ctypes.c_void_p(t.data_ptr()) for t in ts]


def _noalloc(L, dims, dev, x, tol, maxiter):
    it, rr = ctypes.c_int(), ctypes.c_double()
    rc = L.hs_pcg_solve_noalloc(*dims, *_ptrs(dev + [x]), tol, maxiter, None, ctypes.byref(it), ctypes.byref(rr))
    assert rc == 0, L.hs_last_error(None)
    return it.value, rr.value


def _allocating(L, dims, dev, x, tol, maxiter):
    h = ctypes.c_void_p()
    assert L.hs_pcg_create(*dims, 0, ctypes.byref(h)) == 0, L.hs_last_error(None)
    try:
        it, rr = ctypes.c_int(), ctypes.c_double()
        assert L.hs_pcg_solve(h, *_ptrs(dev + [x]), tol, maxiter, None, ctypes.byref(it), ctypes.byref(rr)) == 0
        return it.value, rr.value
    finally:
        L.hs_pcg_destroy(h)


# (30, 20, 14): a ragged grid; (62, 62, 62): (nx+2)(ny+2)(nz+2) = 262144, exactly the static scratch's limit
@pytest.mark.parametrize("dims", [(30, 20, 14), (62, 62, 62)])
def test_noalloc_matches_allocating_solve_on_consecutive_calls(dims):
    import torch
    L = _lib()
    for seed in (11, 12):  # two calls in a row, different systems
        coef, b = _system(*dims, seed)
        dev = [torch.tensor(a, device="cuda") for a in coef + [b]]
        x_ref = torch.zeros_like(dev[3])
        x_na = torch.full_like(dev[3], -3.0)  # stale values must be overwritten
        it1, rr1 = _allocating(L, dims, dev, x_ref, 1e-8, 800)
        it2, rr2 = _noalloc(L, dims, dev, x_na, 1e-8, 800)
        a, r = x_na.cpu().numpy(), x_ref.cpu().numpy()
        assert it1 == it2 > 0
        assert np.linalg.norm(a - r) <= 1e-9 * np.linalg.norm(r)
        assert abs(rr1 - rr2) <= 1e-9 * max(rr1, 1e-300)


def test_noalloc_matches_oracle():
    """Directly against the oracle's HYPRE-rule CG on the same (symmetric
    positive definite) system: the iteration counts within one, x within
    1e-9 (the oracle's sums run in another order, which moves the iterates at
    round-off level)."""
    import torch
    from oracle import oracle
    L = _lib()
    dims = (33, 17, 9)
    coef, b = _system(*dims, 21, symmetric=True)
    dev = [torch.tensor(a, device="cuda") for a in coef + [b]]
    x = torch.zeros_like(dev[3])
    it, rr = _noalloc(L, dims, dev, x, 1e-10, 2000)
    xo, io, ro = oracle.pcg_solve(*dims, *coef, b, tol=1e-10, maxiter=2000)
    assert abs(it - io) <= 1
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-9 * np.linalg.norm(xo)
    assert abs(rr - ro) <= 1e-6 * max(ro, 1e-30) + 1e-14


def test_noalloc_leaves_free_memory_unchanged():
    """After one warm-up call (which loads the library's module on this device
    if nothing else has), further calls change nothing in the device's free
    memory: the scratch is the static array, nothing is allocated."""
    import torch
    L = _lib()
    dims = (40, 30, 20)
    coef, b = _system(*dims, 31)
    dev = [torch.tensor(a, device="cuda") for a in coef + [b]]
    x = torch.zeros_like(dev[3])
    _noalloc(L, dims, dev, x, 1e-8, 500)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _noalloc(L, dims, dev, x, 1e-8, 500)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    L = _lib()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    it, rr = ctypes.c_int(), ctypes.c_double()
    # 63 x 62 x 62: one padded row over the limit
    for dims in ((100, 100, 100), (63, 62, 62)):
        rc = L.hs_pcg_solve_noalloc(*dims, p, p, p, p, p, 1e-5, 10, None, ctypes.byref(it), ctypes.byref(rr))
        assert rc == -1  # HS_ERR_ARG
        assert b"static scratch" in L.hs_last_error(None)
