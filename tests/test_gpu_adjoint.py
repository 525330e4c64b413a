"""Conjugate-heat-transfer energy solve and its adjoint (hs_cht_*):
GPU forward and adjoint against the FP64 CPU oracle, the adjoint gradient
against central finite differences (seeded q directions, every k region), and the
torch.autograd.Function harness."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed=7):
    from hsolver_b200 import cases
    return cases.channel(40, 20, 16, cases.place_blocks((40, 20, 16), 4, 3, 6, seed=seed))


def _setup(steps=5, tol=1e-14):
    import hsolver_b200
    from hsolver_b200.adjoint import ChtProblem
    from oracle import oracle
    deck = _case()
    g = hsolver_b200.Solver(deck)
    g.init()
    g.step(steps)
    prob = ChtProblem(g, k_fluid=1.0, tol=tol, maxiter=20000)
    o = oracle.OracleCase(deck)
    ctype, region = o.cell_types()
    rng = np.random.default_rng(3)
    k = rng.uniform(10.0, 1000.0, prob.nreg)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, ctype.size) * 1e4, 0.0)
    return g, prob, o, ctype, region, k, q


def _grid(o, axis):
    from oracle import oracle
    n = o.dims[axis] + 1
    out = np.empty(n, np.float64)
    assert oracle.lib().or_get_grid(o.h, axis, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == 0
    return out


def test_forward_and_adjoint_match_oracle():
    from oracle import oracle
    g, prob, o, ctype, region, k, q = _setup(tol=1e-13)
    J, T = prob.forward(k, q, want_T=True)
    dq, dk = prob.gradient()
    ug, vg, wg = prob.velocities()
    assert np.abs(ug).max() > 0  # a real flow is frozen in
    kcell = np.where(ctype == 1, k[np.maximum(region, 0)], 1.0)
    ref = oracle.cht_solve(_grid(o, 0), _grid(o, 1), _grid(o, 2), ctype, region, kcell, q, ug, vg, wg,
                           Tb=293.0, tol=1e-13, nreg=prob.nreg)
    assert np.linalg.norm(T - ref["T"]) / np.linalg.norm(ref["T"]) < 1e-10
    assert abs(J - ref["J"]) / ref["J"] < 1e-10
    assert np.linalg.norm(dq - ref["dJdq"]) / np.linalg.norm(ref["dJdq"]) < 1e-8
    assert np.linalg.norm(dk - ref["dJdk"]) / np.linalg.norm(ref["dJdk"]) < 1e-8
    assert np.all(dq[ctype == 0] == 0)


def test_adjoint_gradient_vs_central_differences():
    """dJ/dq along 8 seeded directions (relative step 1e-4) and dJ/dk_b per
    region (relative step 1e-3).  The forward solve stops at a relative
    residual of 1e-14, which leaves ~1e-13 relative noise in J; J moves by
    only ~1e-3 of itself per unit relative change of k, so smaller steps
    drown in that noise, while the central-difference truncation at these
    steps is below 1e-6."""
    g, prob, o, ctype, region, k, q = _setup()
    prob.forward(k, q)
    dq, dk = prob.gradient()
    rng = np.random.default_rng(11)
    solid = ctype == 1
    worst_q = 0.0
    h = 1e-4
    for _ in range(8):
        d = np.where(solid, rng.standard_normal(q.size) * q, 0.0)
        fd = (prob.forward(k, q + h * d) - prob.forward(k, q - h * d)) / (2 * h)
        worst_q = max(worst_q, abs(fd - np.dot(dq, d)) / abs(fd))
    worst_k = 0.0
    h = 1e-3
    for b in range(k.size):
        kp, km = k.copy(), k.copy()
        kp[b] *= 1 + h
        km[b] *= 1 - h
        fd = (prob.forward(kp, q) - prob.forward(km, q)) / (2 * h * k[b])
        worst_k = max(worst_k, abs(fd - dk[b]) / abs(fd))
    assert worst_q <= 1e-5, worst_q
    assert worst_k <= 1e-5, worst_k


def test_autograd_function_matches_adjoint():
    import torch
    from hsolver_b200.adjoint import objective_function
    g, prob, o, ctype, region, k, q = _setup(tol=1e-12)
    Obj = objective_function()
    qt = torch.tensor(q, requires_grad=True)
    kt = torch.tensor(k, requires_grad=True)
    J = Obj.apply(qt, kt, prob)
    J.backward()
    prob.forward(k, q)
    dq, dk = prob.gradient()
    assert np.allclose(qt.grad.numpy(), dq, rtol=1e-12, atol=0)
    assert np.allclose(kt.grad.numpy(), dk, rtol=1e-12, atol=0)
    assert prob.last["adjoint_iters"] <= 1.5 * prob.last["forward_iters"] + 5
