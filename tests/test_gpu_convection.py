"""Hybrid and QUICK momentum convection and Boussinesq buoyancy on the GPU
against the CPU oracle (or_ch_*, which the CPU tests pin to the published
QUICK and hybrid rules and to the hydrostatic balance): the momentum sweeps
bit for bit (the buoyancy term from a set, non-uniform temperature), full
outer steps with tight inner tolerances, the converged state of a heated,
buoyant channel in both precisions, and the hydrostatic pressure of a uniform
temperature excess on a stretched grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FACE = ["u", "v", "w"]
OKEYS = ("re", "pr", "u_in", "t_in", "alpha_u", "alpha_p", "alpha_t", "mom_sweeps", "p_tol", "p_maxiter", "t_tol",
         "t_maxiter", "conv", "g_axis", "ri")


def _deck(zs=None):
    from hsolver_b200 import cases
    xs, ys = cases.uniform(24, 2.0), cases.uniform(12, 1.0)
    return cases.deck_text(xs, ys, cases.uniform(12, 1.0) if zs is None else zs, blocks=[(9, 12, 1, 4, 5, 8)])


def _pair(deck, q_on=True, **kw):
    import hsolver_b200
    from oracle import oracle
    g = hsolver_b200.Channel(deck, **kw)
    o = oracle.ChannelCase(deck, **{k: v for k, v in kw.items() if k in OKEYS})
    n = o.dims[0] * o.dims[1] * o.dims[2]
    ctype, _ = oracle.OracleCase(deck).cell_types()
    rng = np.random.default_rng(7)
    k = rng.uniform(10.0, 1000.0, o.nreg)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, n), 0.0) if q_on else np.zeros(n)
    g.set_solid(k, q)
    o.set_solid(k, q)
    g.init()
    o.init()
    return g, o, ctype


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("conv,ri,g_axis", [(1, 0.0, 2), (2, 0.0, 2), (0, 1.5, 1), (2, 1.5, 2)])
def test_momentum_sweeps_bit_exact(conv, ri, g_axis):
    g, o, ctype = _pair(_deck(), re=150.0, conv=conv, ri=ri, g_axis=g_axis)
    T = np.random.default_rng(3).uniform(0.0, 2.0, ctype.size)  # a temperature field for the buoyancy term
    g.set_field("T", T)
    o.set_field("T", T)
    for step in range(3):
        gs = g.step(1, flags=3)
        o.step(1, pressure=False, energy=False)
        for name in FACE + ["u_star", "v_star", "w_star", "d_u", "d_v", "d_w"]:
            a, b = g.field(name), o.field(name)
            assert np.array_equal(a, b), (step, name, np.abs(a - b).max())
        ores = o.stats()["res"]
        for x in range(3):
            assert abs(gs["res"][x] - ores[x]) <= 1e-12 * max(ores[x], 1e-300)


@pytest.mark.parametrize("conv", [1, 2])
def test_outer_steps_match_oracle(conv):
    g, o, _ = _pair(_deck(), re=150.0, conv=conv, ri=1.0, g_axis=2, p_tol=1e-13, p_maxiter=5000, t_tol=1e-13,
                    t_maxiter=5000)
    for step in range(5):
        gs = g.step(1)
        o.step(1)
        os_ = o.stats()
        for name in FACE + ["p", "T", "p_prime"]:
            assert _rel(g.field(name), o.field(name)) < 1e-9, (step, name)
        for x in range(5):
            assert abs(gs["res"][x] - os_["res"][x]) <= 1e-8 * max(os_["res"][x], 1e-300), (step, x)


@pytest.mark.parametrize("precision", [0, 1])
def test_buoyant_quick_channel_converges_to_the_oracle_state(precision):
    """QUICK with buoyancy on (the heated blocks drive a plume along +z): the
    GPU at a global residual of 1e-7, in FP64 and in the mixed form, against
    the oracle run for the same number of steps."""
    g, o, _ = _pair(_deck(), re=150.0, conv=2, ri=2.0, g_axis=2, precision=precision)
    ok, steps, st = g.solve_to(1e-7, 4000)
    assert ok, st
    o.step(steps)
    assert o.stats()["global"] <= 1e-7 * 1.5
    for name in FACE + ["p", "T"]:
        assert _rel(g.field(name), o.field(name)) < 1e-6, name


def test_uniform_temperature_excess_is_hydrostatic():
    from hsolver_b200 import cases
    zs = cases.tanh_clustered(12, 1.0, 6.0, 2.0 / 24)
    deck = _deck(zs)
    ri = 2.0
    fields = []
    for r in (0.0, ri):
        g, _, ctype = _pair(deck, q_on=False, re=100.0, ri=r, g_axis=2, p_tol=1e-11, p_maxiter=5000)
        g.set_field("T", np.ones(ctype.size))  # t_in = 0
        st = g.step(500, flags=2)
        assert st["global"] < 1e-11
        fields.append({n: g.field(n) for n in FACE + ["p"]})
    for f in FACE:
        assert _rel(fields[1][f], fields[0][f]) <= 1e-10, f
    zc = 0.5 * (zs[:-1] + zs[1:])
    Nz, Ny, Nx = 12, 12, 24
    dev = fields[1]["p"] - fields[0]["p"] - ri * np.broadcast_to(zc[:, None, None], (Nz, Ny, Nx)).ravel()
    assert np.ptp(dev[ctype == 0]) <= 1e-9 * ri


def test_quick_sweeps_bit_exact_on_a_stretched_grid():
    """QUICK's weights come from the node positions: on a tanh-stretched grid
    in y and z (maximum aspect ratio 8) they are not the uniform 6/8, 3/8,
    -1/8, and the GPU's host-built tables must match the oracle's bit for
    bit through the sweeps."""
    from hsolver_b200 import cases
    xs = cases.uniform(24, 2.0)
    ys = cases.tanh_clustered(12, 1.0, 8.0, 2.0 / 24)
    zs = cases.tanh_clustered(12, 1.0, 8.0, 2.0 / 24)
    deck = cases.deck_text(xs, ys, zs, blocks=[(9, 12, 1, 4, 5, 8)])
    g, o, ctype = _pair(deck, re=150.0, conv=2, ri=0.8, g_axis=1)
    T = np.random.default_rng(8).uniform(0.0, 2.0, ctype.size)
    g.set_field("T", T)
    o.set_field("T", T)
    for step in range(3):
        g.step(1, flags=3)
        o.step(1, pressure=False, energy=False)
        for name in FACE + ["u_star", "v_star", "w_star", "d_u", "d_v", "d_w"]:
            a, b = g.field(name), o.field(name)
            assert np.array_equal(a, b), (step, name, np.abs(a - b).max())
