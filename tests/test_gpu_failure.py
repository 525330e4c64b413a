"""Failure paths of the channel solver through the C ABI, made on the host:
a NaN written into the state through hs_channel_set_field makes the next
hs_channel_step return HS_ERR_DIVERGED (every kernel only computes with the
NaN; the iteration limits bound the inner solves), and hs_channel_solve_to
with too few outer steps returns HS_ERR_MAXITER.  The context stays usable
after both: a fresh solver on the same device steps normally."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _channel(**kw):
    import hsolver_b200
    from hsolver_b200 import cases
    deck = cases.channel(24, 12, 12, [(9, 12, 1, 4, 5, 8)])
    g = hsolver_b200.Channel(deck, re=100.0, **kw)
    ctype, _ = hsolver_b200.Case(deck).cell_types()
    g.set_solid(np.full(g.nblocks, 100.0), np.where(ctype == 1, 1.0, 0.0))
    g.init()
    return g


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_in_the_state_reports_diverged(precision):
    import hsolver_b200
    g = _channel(precision=precision, p_maxiter=50, t_maxiter=20)
    g.step(2)
    u = g.field("u")
    u[u.size // 2] = np.nan
    g.set_field("u", u)
    with pytest.raises(hsolver_b200.HsError) as e:
        g.step(1)
    assert e.value.code == -7  # HS_ERR_DIVERGED
    g.close()
    h = _channel(precision=precision)
    st = h.step(3)
    assert np.isfinite(st["res"]).all() and st["iter"] == 3
    h.close()


def test_solve_to_reports_maxiter():
    import hsolver_b200
    g = _channel()
    L = hsolver_b200.load()
    steps = ctypes.c_int()
    st = hsolver_b200.ChannelStats()
    rc = L.hs_channel_solve_to(g.h, 1e-12, 8, ctypes.byref(steps), ctypes.byref(st))
    assert rc == -9  # HS_ERR_MAXITER
    assert steps.value == 8 and st.iter == 8 and st.global_ > 1e-12
    assert b"above tolerance" in L.hs_last_error(None)
    ok, n, _ = g.solve_to(1e-6, 2000)  # the same solver continues to convergence
    assert ok and n > 0
    g.close()
