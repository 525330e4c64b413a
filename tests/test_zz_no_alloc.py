"""hs_pcg_solve_noalloc: the pressure-correction solve for callers that cannot
allocate device memory while they run (their GPU memory belongs to their own
arena, or cudaMalloc/cudaFree would synchronise the device in the middle of
their loop).  It must give the same answer as the allocating hs_pcg_solve,
call after call, although every call reuses one static scratch array.

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    shape = (nz + 2, ny + 2, nx + 2)
    unknown = np.zeros(shape, bool)
    unknown[1:-1, 1:-1, 1:-1] = True
    unknown[2:4, 2:5, 3:7] = False  # a block of non-unknowns
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


def test_noalloc_matches_allocating_solve_on_consecutive_calls():
    import torch
    L = _lib()
    dims = (30, 20, 14)
    h = ctypes.c_void_p()
    assert L.hs_pcg_create(*dims, 0, ctypes.byref(h)) == 0, L.hs_last_error(None)
    try:
        for seed in (11, 12):  # two calls in a row, different systems
            coef, b = _system(*dims, seed)
            dev = [torch.tensor(a, device="cuda") for a in coef + [b]]
            x_ref = torch.zeros_like(dev[3])
            x_na = torch.full_like(dev[3], -3.0)  # stale values must be overwritten
            it1, rr1 = ctypes.c_int(), ctypes.c_double()
            it2, rr2 = ctypes.c_int(), ctypes.c_double()
            assert L.hs_pcg_solve(h, *_ptrs(dev + [x_ref]), 1e-8, 500, None, ctypes.byref(it1), ctypes.byref(rr1)) == 0
            rc = L.hs_pcg_solve_noalloc(*dims, *_ptrs(dev + [x_na]), 1e-8, 500, None, ctypes.byref(it2),
                                        ctypes.byref(rr2))
            assert rc == 0, L.hs_last_error(None)
            a, r = x_na.cpu().numpy(), x_ref.cpu().numpy()
            assert it1.value == it2.value > 0
            assert np.linalg.norm(a - r) <= 1e-9 * np.linalg.norm(r)
            assert abs(rr1.value - rr2.value) <= 1e-9 * max(rr1.value, 1e-300)
    finally:
        L.hs_pcg_destroy(h)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    L = _lib()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    it, rr = ctypes.c_int(), ctypes.c_double()
    rc = L.hs_pcg_solve_noalloc(100, 100, 100, p, p, p, p, p, 1e-5, 10, None, ctypes.byref(it), ctypes.byref(rr))
    assert rc == -1  # HS_ERR_ARG
    assert b"static scratch" in L.hs_last_error(None)
