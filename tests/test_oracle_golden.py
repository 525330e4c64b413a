"""The CPU oracle against golden fixtures produced by the reference's own
sources (tests/golden/make_golden.py): bit-exact, every state array."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, read_deck

FIELD_ARRAYS = ["u_star", "v_star", "w_star", "up", "vp", "wp", "p_temp", "t_temp", "ux", "uy", "uz", "p", "t"]


def _steps(npz):
    return sorted({int(k.split("/")[0]) for k in npz.files})


@pytest.mark.parametrize("deck", ["small", "inner", "quirk"])
def test_oracle_matches_reference_full_state(oracle_mod, deck):
    g = np.load(os.path.join(GOLDEN, "golden_%s.npz" % deck))
    oc = oracle_mod.OracleCase(read_deck(deck))
    oc.init()
    done = 0
    for s in _steps(g):
        oc.step(s - done)
        done = s
        for name in FIELD_ARRAYS:
            ref = g["%d/%s" % (s, name)]
            got = oc.field(name)
            assert ref.shape == got.shape, name
            assert np.array_equal(ref, got), "%s differs at step %d (max |d| %g)" % (name, s, np.max(np.abs(ref - got)))
        assert np.array_equal(g["%d/solid.t_temp" % s], oc.solid(0)), "solid t_temp step %d" % s
        assert np.array_equal(g["%d/solid.t" % s], oc.solid(0, "t")), "solid t step %d" % s
        em = g["%d/fluid.empty" % s].astype(np.uint8)
        assert np.array_equal(em, oc.fluid_empty())
        ids = g["%d/id" % s]
        assert np.array_equal(ids[em == 0], oc.row_ids()[em == 0])
        assert int(g["%d/pcg_iters" % s][0]) == oc.stats()["pcg_iters"]
        meta = g["%d/fluid.meta" % s].astype(np.int64)
        assert tuple(meta) == oc.meta


@pytest.mark.parametrize("deck", ["small", "inner", "quirk"])
def test_oracle_interface_lists_match_reference(oracle_mod, deck):
    """The fluid<->solid temperature exchange pairs equal the reference's
    t_boundary / t_halo lists (fluid_solver.h:983-1006, mobs_solver.h:147-167)."""
    g = np.load(os.path.join(GOLDEN, "golden_%s.npz" % deck))
    s = _steps(g)[0]
    oc = oracle_mod.OracleCase(read_deck(deck))
    pairs = oc.swap_pairs()
    assert np.array_equal(pairs[:, 0], g["%d/fluid.t_boundary" % s])
    assert np.array_equal(pairs[:, 1], g["%d/fluid.t_halo" % s])
    assert np.array_equal(pairs[:, 2], g["%d/solid.t_boundary" % s])
    assert np.array_equal(pairs[:, 3], g["%d/solid.t_halo" % s])


def test_oracle_matches_reference_digests(oracle_mod):
    """Larger decks (config-1 channel, the stretched config-3 grid, the
    reference's own example13.in): SHA-256 of every FP64 array."""
    with open(os.path.join(GOLDEN, "golden_digests.json")) as f:
        dig = json.load(f)
    for deck, per_step in dig.items():
        oc = oracle_mod.OracleCase(read_deck(deck))
        oc.init()
        done = 0
        for s in sorted(per_step, key=int):
            oc.step(int(s) - done)
            done = int(s)
            ent = per_step[s]
            for name in FIELD_ARRAYS:
                if name not in ent:
                    continue
                got = oc.field(name)
                assert hashlib.sha256(got.tobytes()).hexdigest() == ent[name]["sha256"], (deck, s, name)
            st = ent.get("solid.t_temp")
            if st:
                assert hashlib.sha256(oc.solid(0).tobytes()).hexdigest() == st["sha256"], (deck, s, "solid")
            assert oc.stats()["pcg_iters"] == ent["pcg_iters"]


def test_deck_parser_drops_value_without_trailing_comma(oracle_mod):
    """mesh/mesh.cpp:1677: `lineiss >> value >> spliter` drops a last value
    with no separator; quirk.in's x-line ends in `2.2` without a comma."""
    oc = oracle_mod.OracleCase(read_deck("quirk"))
    assert oc.dims == (9, 6, 6)


def test_oracle_reads_deck_lines_of_any_length():
    """A 1000-cell axis puts ~8 kB on one deck line (more than the oracle's
    former 4 kB line buffer held); the oracle reads it
    whole, as std::getline does in the reference (mesh/mesh.cpp:1673), and
    agrees with the product's case model."""
    import numpy as np
    from hsolver_b200 import cases
    from oracle import oracle
    import hsolver_b200
    deck = cases.deck_text(np.linspace(0.0, 2.0, 1001), np.linspace(0.0, 1.0, 3), np.linspace(0.0, 1.0, 3),
                           blocks=[(500, 510, 1, 1, 1, 1)])
    assert max(len(x) for x in deck.splitlines()) > 4096
    o = oracle.OracleCase(deck)
    assert tuple(o.dims) == (1000, 2, 2)
    assert tuple(hsolver_b200.Case(deck).dims) == (1000, 2, 2)
