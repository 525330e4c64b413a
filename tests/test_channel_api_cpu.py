"""Argument checks of the channel C ABI that need no GPU: parameters and
decks are rejected with the documented codes before any device work."""
import ctypes

import pytest


def _L():
    import hsolver_b200
    L = hsolver_b200.load()
    hsolver_b200._channel_api(L)
    return hsolver_b200, L


def _deck():
    from hsolver_b200 import cases
    return cases.channel(12, 6, 6, [(5, 7, 1, 3, 2, 4)])


@pytest.mark.parametrize("field,value", [("re", 0.0), ("pr", -1.0), ("alpha_u", 0.0), ("alpha_u", 1.5),
                                         ("alpha_p", 0.0), ("alpha_t", 2.0), ("mom_sweeps", 0), ("p_tol", 0.0),
                                         ("t_tol", -1.0), ("precision", 2), ("p_maxiter", -1)])
def test_invalid_parameters_are_rejected(field, value):
    hs, L = _L()
    p = hs.channel_params(**{field: value})
    h = ctypes.c_void_p()
    rc = L.hs_channel_create(_deck().encode(), ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == -1, (field, value, rc)  # HS_ERR_ARG
    assert not h.value
    assert b"invalid channel parameters" in L.hs_last_error(None)


def test_bad_deck_is_rejected():
    hs, L = _L()
    p = hs.channel_params()
    h = ctypes.c_void_p()
    assert L.hs_channel_create(b"not a deck", ctypes.byref(p), 0, ctypes.byref(h)) == -2  # HS_ERR_DECK
    assert L.hs_channel_create(None, ctypes.byref(p), 0, ctypes.byref(h)) == -1


def test_null_handle_calls_fail_cleanly():
    hs, L = _L()
    st = hs.ChannelStats()
    assert L.hs_channel_step(None, 1, 0, ctypes.byref(st)) == -1
    assert L.hs_channel_init(None) == -1
    n = ctypes.c_longlong()
    assert L.hs_channel_field_size(None, 0, ctypes.byref(n)) == -1
    L.hs_channel_destroy(None)


def test_defaults():
    hs, L = _L()
    p = hs.channel_params()
    assert (p.re, p.pr, p.u_in, p.alpha_u, p.alpha_p, p.alpha_t) == (100.0, 0.71, 1.0, 0.7, 0.3, 0.9)
    assert (p.mom_sweeps, p.p_tol, p.p_maxiter, p.precision, p.p_precond) == (2, 1e-8, 1000, 0, 1)
