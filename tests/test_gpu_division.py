"""The sweeps divide by per-axis geometry with a precomputed reciprocal and
one FMA correction (Markstein's method).  It must give IEEE a/b bit for bit;
checked on the GPU over random and adversarial operands."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(a, b):
    import hsolver_b200
    L = hsolver_b200.load()
    L.hs_check_division.restype = ctypes.c_longlong
    L.hs_check_division.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2 + [ctypes.c_longlong]
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return L.hs_check_division(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size)


def test_random_operands_bit_exact():
    rng = np.random.default_rng(0)
    n = 4_000_000
    a = rng.uniform(-1e3, 1e3, n) * 10.0 ** rng.integers(-8, 8, n)
    b = rng.uniform(1e-4, 1.0, n) * 10.0 ** rng.integers(-3, 3, n)
    assert _check(a, b) == 0


def test_adversarial_significands_bit_exact():
    rng = np.random.default_rng(1)
    n = 4_000_000
    # divisors with significands at the ends of the binade, dividends of all kinds
    m = np.concatenate([1 + rng.integers(0, 2 ** 20, n // 2) * 2.0 ** -52, 2 - rng.integers(1, 2 ** 20, n // 2) * 2.0 ** -52])
    b = m * 2.0 ** rng.integers(-10, 10, n)
    a = np.concatenate([rng.uniform(1, 2, n // 2), 1 + rng.integers(0, 2 ** 26, n // 2) * 2.0 ** -52]) * 2.0 ** rng.integers(-10, 10, n)
    assert _check(a, b) == 0


def test_geometry_divisions_of_the_decks_bit_exact():
    """Every (numerator-like, spacing) pair the energy sweep sees on the
    fixture grids: alpha*(T1+T2) over the cell spacings."""
    from conftest import read_deck
    from oracle import oracle
    rng = np.random.default_rng(2)
    b = []
    for deck in ["example13", "example21", "config3"]:
        o = oracle.OracleCase(read_deck(deck))
        for ax in range(3):
            g = np.diff(o_grid(o, ax))
            s = (g[1:] + g[:-1]) / 2.0
            b.append(s)
    b = np.concatenate(b)
    bb = np.repeat(b, 2000)
    a = 0.001 * rng.uniform(500, 700, bb.size)
    assert _check(a, bb) == 0
    assert _check(a / bb, bb) == 0


def o_grid(o, axis):
    from oracle import oracle
    n = o.dims[axis] + 1
    out = np.empty(n, np.float64)
    assert oracle.lib().or_get_grid(o.h, axis, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == 0
    return out
