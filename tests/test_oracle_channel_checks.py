"""The oracle's checks of a step solved elsewhere (or_ch_step_given,
or_ch_energy_residual), against the oracle's own step on the CPU: a step
given the p' the oracle itself solved reproduces that step bit for bit with
the solve's residual, and the energy residual of the relaxed step's
unrelaxed temperature is the solve's."""
import numpy as np


def _case(**kw):
    from hsolver_b200 import cases
    from oracle import oracle
    deck = cases.channel(24, 12, 12, [(9, 12, 1, 4, 5, 8)])
    o = oracle.ChannelCase(deck, re=100.0, **kw)
    ctype, _ = oracle.OracleCase(deck).cell_types()
    o.set_solid(np.full(o.nreg, 50.0), np.where(ctype == 1, 1.0, 0.0))
    o.init()
    return o


def test_step_given_the_oracles_own_pprime_reproduces_its_step():
    from oracle import oracle
    kw = dict(p_tol=1e-12, p_maxiter=20000, t_tol=1e-12, t_maxiter=20000)
    a, b = _case(**kw), _case(**kw)
    for _ in range(2):
        a.step(1, energy=False)
        b.step(1, energy=False)
    a.step(1, energy=False)
    rel = oracle.channel_step_given(b, a.field("p_prime"))
    assert 0 < rel < 1e-11
    for name in ("u", "v", "w", "p", "p_prime", "u_star", "d_u"):
        assert np.array_equal(a.field(name), b.field(name)), name


def test_energy_residual_of_a_solved_step():
    from oracle import oracle
    o = _case(p_tol=1e-12, p_maxiter=20000, t_tol=1e-12, t_maxiter=20000)
    o.step(2)
    t0 = o.field("T")
    o.step(1)
    t1 = o.field("T")
    tt = t0 + (t1 - t0) / 0.9  # the unrelaxed solve (alpha_t = 0.9)
    r, bn = oracle.channel_energy_residual(o, tt)
    assert bn > 0 and r <= 1e-10 * bn
    r0, _ = oracle.channel_energy_residual(o, t0)
    assert r0 > 1e3 * r
