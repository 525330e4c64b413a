"""C-ABI library checks that need no GPU: it loads, exports every symbol the
header declares, rejects bad decks with the documented status, and its host
case model (masks, regions, boxes, interface pairs) is bit-exact with the
oracle on every fixture deck and the seeded configs."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO, read_deck

HEADER = os.path.join(REPO, "include", "hsolver_b200.h")


def _lib():
    import hsolver_b200
    return hsolver_b200.load()


def test_library_exports_every_declared_symbol():
    L = _lib()
    src = open(HEADER).read()
    names = sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w ]*?[\s\*]+)(hs_\w+)\s*\(", src, re.M)))
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("deck,code", [
    ("ygrid = 0,1,\nzgrid = 0,1,\nmobs =\nwalls =\nholes =\n", -2),                         # no xgrid
    ("; comment\nxgrid = 0,1,2,\nygrid = 0,1,2,\nzgrid = 0,1,2,\nmobs =\nwalls =\nholes =\n", -2),  # xgrid not at byte 0
    ("xgrid = 0,1,2,\nygrid = 0,1,2,\nzgrid = 0,1,2,\nmobs =\n 1,2,\nwalls =\nholes =\n", -2),  # short mobs line
    ("xgrid = 0,1,2,3,\nygrid = 0,1,2,3,\nzgrid = 0,1,2,3,\nmobs =\n 2,2,1,3,1,3,\nwalls =\nholes =\n", -3),  # two fluid regions
])
def test_bad_decks_rejected(deck, code):
    import hsolver_b200
    with pytest.raises(hsolver_b200.HsError) as e:
        hsolver_b200.Case(deck)
    assert e.value.code == code


def _compare_case(oracle_mod, text):
    import hsolver_b200
    c = hsolver_b200.Case(text)
    o = oracle_mod.OracleCase(text)
    assert c.dims == o.dims
    assert c.meta == o.meta
    t1, r1 = c.cell_types()
    t2, r2 = o.cell_types()
    assert np.array_equal(t1, t2) and np.array_equal(r1, r2)
    assert np.array_equal(c.fluid_empty(), o.fluid_empty())
    assert c.nsolid == o.nsolid
    for r in range(c.nsolid):
        assert c.solid_meta(r) == o.solid_meta(r)
    assert np.array_equal(c.interface(), o.swap_pairs())


@pytest.mark.parametrize("deck", ["small", "inner", "quirk", "config1", "config3", "example13", "example21"])
def test_case_model_matches_oracle_on_fixture_decks(oracle_mod, deck):
    _compare_case(oracle_mod, read_deck(deck))


@pytest.mark.parametrize("cfg", ["config2", "config4"])
def test_case_model_matches_oracle_on_seeded_configs(oracle_mod, cfg):
    from hsolver_b200 import cases
    _compare_case(oracle_mod, cases.CONFIGS[cfg](seed=3))


def test_cell_mask_matches_reference_dump():
    """Cell-type mask bit-exact against the reference's own LocalCell::isEmpty
    (tests/golden, produced by the reference sources)."""
    import hsolver_b200
    from conftest import GOLDEN
    for deck in ["small", "inner", "quirk"]:
        g = np.load(os.path.join(GOLDEN, "golden_%s.npz" % deck))
        step = sorted({int(k.split("/")[0]) for k in g.files})[0]
        c = hsolver_b200.Case(read_deck(deck))
        assert np.array_equal(c.fluid_empty(), g["%d/fluid.empty" % step].astype(np.uint8))
        assert np.array_equal(c.interface()[:, 0], g["%d/fluid.t_boundary" % step])
        assert np.array_equal(c.interface()[:, 1], g["%d/fluid.t_halo" % step])
