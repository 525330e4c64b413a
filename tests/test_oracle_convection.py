"""The channel oracle's momentum convection schemes and Boussinesq buoyancy,
pinned independently of the restatement they check the GPU against:

* QUICK (Leonard 1979): on a uniform grid the face value is
  6/8 upwind + 3/8 downwind - 1/8 far upwind; on any grid the weights are
  those of the quadratic through the three nodes, so they reproduce every
  quadratic exactly; where the far-upwind node is off the grid the face takes
  the upwind value;
* hybrid (Spalding 1972): central differencing below a cell Peclet number of
  2, upwind without diffusion above it;
* buoyancy: a uniform temperature excess is a uniform body force, which a
  hydrostatic pressure gradient balances exactly: the converged velocities
  are those without buoyancy and p grows by ri (T - t_in) z over the cell
  centres, on a stretched grid;
* QUICK by deferred correction converges (no residual floor) on a heated
  channel and moves the solution by a few percent from upwind's.
"""
import numpy as np
import pytest

from hsolver_b200 import cases
from oracle import oracle


def test_quick_weights_on_a_uniform_grid():
    pts = np.linspace(0.0, 2.0, 17)
    for kind in (0, 1):
        for e in range(3, 13):
            w = oracle.quick_weights(pts, kind, e)
            assert np.allclose(w, [-1 / 8, 6 / 8, 3 / 8, -1 / 8, 6 / 8, 3 / 8], rtol=0, atol=1e-14), (kind, e, w)


def test_quick_weights_reproduce_quadratics():
    rng = np.random.default_rng(5)
    n = 20
    pts = np.concatenate([[0.0], np.cumsum(rng.uniform(0.3, 1.7, n))])
    centres = 0.5 * (pts[:-1] + pts[1:])
    for kind in (0, 1):
        nodes = pts if kind else centres
        for e in range(0, n + 1 if kind == 0 else n):
            w = oracle.quick_weights(pts, kind, e)
            xf = 0.5 * (pts[e] + pts[e + 1]) if kind else pts[e]
            lo = e if kind else e - 1
            for d, (iuu, iu, idn) in enumerate([(lo - 1, lo, lo + 1), (lo + 2, lo + 1, lo)]):
                ww = w[3 * d:3 * d + 3]
                if min(iuu, iu, idn) < 0 or max(iuu, iu, idn) >= len(nodes):
                    assert list(ww) == [0.0, 1.0, 0.0]
                    continue
                x = nodes[[iuu, iu, idn]]
                for p in range(3):
                    assert abs(ww @ x ** p - xf ** p) <= 1e-11 * max(1.0, abs(xf) ** p), (kind, e, d, p)


def test_hybrid_rule():
    D = 1.0
    for F in (-1.5, -0.3, 0.0, 0.7, 1.9):  # |Pe| < 2: central differencing
        assert oracle.neighbour_coefficient(1, D, F, 1) == pytest.approx(D - F / 2)
        assert oracle.neighbour_coefficient(1, D, F, 0) == pytest.approx(D + F / 2)
    for F in (-7.0, -2.5, 2.5, 7.0):  # |Pe| > 2: upwind, no diffusion
        assert oracle.neighbour_coefficient(1, D, F, 1) == pytest.approx(max(-F, 0.0))
        assert oracle.neighbour_coefficient(1, D, F, 0) == pytest.approx(max(F, 0.0))
        # the reference's first-order upwind keeps the diffusion
        assert oracle.neighbour_coefficient(0, D, F, 1) == pytest.approx(D + max(-F, 0.0))


def _stretched_deck():
    xs = cases.uniform(24, 2.0)
    ys = cases.uniform(12, 1.0)
    zs = cases.tanh_clustered(12, 1.0, 6.0, 2.0 / 24)
    return deck_with(xs, ys, zs), zs


def deck_with(xs, ys, zs):
    return cases.deck_text(xs, ys, zs, blocks=[(9, 12, 1, 4, 5, 8)])


def _hydro(deck, ri, steps):
    oc = oracle.ChannelCase(deck, re=100.0, ri=ri, g_axis=2, p_tol=1e-11, p_maxiter=5000)
    ctype, _ = oracle.OracleCase(deck).cell_types()
    oc.set_solid(np.full(oc.nreg, 100.0), np.zeros(ctype.size))
    oc.init()
    oc.set_field("T", np.ones(ctype.size))  # t_in = 0: a uniform excess of 1
    oc.step(steps, energy=False)
    return oc, ctype


def test_buoyancy_of_a_uniform_temperature_is_hydrostatic():
    deck, zs = _stretched_deck()
    ri = 2.0
    o0, ctype = _hydro(deck, 0.0, 500)
    o1, _ = _hydro(deck, ri, 500)
    assert o0.stats()["global"] < 1e-12 and o1.stats()["global"] < 1e-12
    for f in ("u", "v", "w"):
        a, b = o0.field(f), o1.field(f)
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(a), f
    zc = 0.5 * (zs[:-1] + zs[1:])
    Nx, Ny, Nz = o0.dims
    dev = o1.field("p") - o0.field("p") - ri * np.broadcast_to(zc[:, None, None], (Nz, Ny, Nx)).ravel()
    fluid = ctype == 0
    assert np.ptp(dev[fluid]) <= 1e-10 * ri


def _heated(conv, steps):
    deck = cases.channel(24, 12, 12, [(9, 12, 1, 4, 5, 8)])
    oc = oracle.ChannelCase(deck, re=200.0, conv=conv, p_tol=1e-10, p_maxiter=5000)
    ctype, _ = oracle.OracleCase(deck).cell_types()
    q = np.where(ctype == 1, 1.0, 0.0)
    oc.set_solid(np.full(oc.nreg, 100.0), q)
    oc.init()
    oc.step(steps)
    return oc


def test_quick_deferred_correction_converges():
    up, qk = _heated(0, 400), _heated(2, 400)
    assert up.stats()["global"] < 1e-8
    assert qk.stats()["global"] < 1e-8
    du = np.linalg.norm(qk.field("u") - up.field("u")) / np.linalg.norm(up.field("u"))
    assert 1e-4 < du < 0.2
