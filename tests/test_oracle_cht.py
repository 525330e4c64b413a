"""The oracle's conjugate-heat-transfer solve and adjoint (or_cht_forward /
or_cht_adjoint) checked by themselves on the CPU: the adjoint gradient
against central finite differences of the oracle's own forward solve, with
no flow and with a frozen flow through the fluid.  The GPU adjoint is
compared with this oracle, so this is the pin of that comparison."""
import ctypes

import numpy as np
import pytest


def _problem(flow):
    from hsolver_b200 import cases
    from oracle import oracle
    deck = cases.channel(20, 10, 8, cases.place_blocks((20, 10, 8), 2, 2, 3, seed=5))
    o = oracle.OracleCase(deck)
    ctype, region = o.cell_types()
    grids = []
    for axis in range(3):
        g = np.empty(o.dims[axis] + 1)
        assert oracle.lib().or_get_grid(o.h, axis, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), g.size) == 0
        grids.append(g)
    Nx, Ny, Nz = (g.size - 1 for g in grids)
    ug, vg, wg = np.zeros((Nz, Ny, Nx + 1)), np.zeros((Nz, Ny + 1, Nx)), np.zeros((Nz + 1, Ny, Nx))
    if flow:
        s = (ctype == 1).reshape(Nz, Ny, Nx)
        ug[:] = 0.05
        ug[:, :, 1:-1][s[:, :, 1:] | s[:, :, :-1]] = 0.0  # no flux through a face that touches a solid
        ug[:, :, 0][s[:, :, 0]] = 0.0
        ug[:, :, -1][s[:, :, -1]] = 0.0
    nreg = int(region.max()) + 1
    rng = np.random.default_rng(3)
    k = rng.uniform(10.0, 1000.0, nreg)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, ctype.size) * 1e4, 0.0)

    def run(kk, qq):
        kcell = np.where(ctype == 1, kk[np.maximum(region, 0)], 1.0)
        return oracle.cht_solve(*grids, ctype, region, kcell, qq, ug.ravel(), vg.ravel(), wg.ravel(),
                                Tb=293.0, tol=1e-15, nreg=nreg)

    return run, ctype, k, q


@pytest.mark.parametrize("flow", [False, True])
def test_oracle_adjoint_vs_central_differences(flow):
    run, ctype, k, q = _problem(flow)
    base = run(k, q)
    assert np.isfinite(base["J"]) and base["J"] > 0.0  # J = (sum over solid T^8 V)^(1/8), not a mean
    rng = np.random.default_rng(11)
    for _ in range(3):
        d = np.where(ctype == 1, rng.standard_normal(q.size) * q, 0.0)
        h = 1e-4
        fd = (run(k, q + h * d)["J"] - run(k, q - h * d)["J"]) / (2 * h)
        assert abs(fd - np.dot(base["dJdq"], d)) <= 1e-6 * abs(fd)
    for b in range(k.size):
        h = 1e-3
        kp, km = k.copy(), k.copy()
        kp[b] *= 1 + h
        km[b] *= 1 - h
        fd = (run(kp, q)["J"] - run(km, q)["J"]) / (2 * h * k[b])
        assert abs(fd - base["dJdk"][b]) <= 1e-5 * abs(fd)
