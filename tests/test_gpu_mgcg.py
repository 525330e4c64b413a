"""HS_PSOLVE_MGCG: CG preconditioned by the FP32 multigrid V-cycle solves the
same pressure-correction system as the reference's CG.  Both solved tightly,
the outer steps agree with the oracle; at the reference tolerance the MG
solve needs far fewer iterations."""
import numpy as np
import pytest

from conftest import read_deck

pytestmark = pytest.mark.gpu

FIELDS = ["u_star", "v_star", "w_star", "p_temp", "t_temp", "p", "t"]


def _rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (n if n > 0 else 1.0)


@pytest.mark.parametrize("deck,steps", [("inner", 4), ("config1", 3), ("example13", 2)])
def test_mgcg_tight_matches_oracle(deck, steps):
    import hsolver_b200
    from oracle import oracle
    text = read_deck(deck)
    g = hsolver_b200.Solver(text, hsolver_b200.default_params(pressure_solver=hsolver_b200.PSOLVE_MGCG,
                                                              pcg_tol=1e-11, pcg_maxiter=500))
    op = oracle.default_params()
    op.pcg_tol = 1e-11
    op.pcg_maxiter = 5000
    o = oracle.OracleCase(text, op)
    g.init()
    o.init()
    for _ in range(steps):
        st = g.step(1, stats=True)
        o.step(1)
        assert st["pcg_relres"] < 1e-11
    for f in FIELDS:
        assert _rel(g.field(f), o.field(f)) < 1e-7, f


def test_mgcg_needs_fewer_iterations():
    import hsolver_b200
    from hsolver_b200 import cases
    deck = cases.config4(0)
    it = {}
    for ps in (hsolver_b200.PSOLVE_CG, hsolver_b200.PSOLVE_MGCG):
        g = hsolver_b200.Solver(deck, hsolver_b200.default_params(pressure_solver=ps))
        g.init()
        g.step(2)
        it[ps] = g.step(1, stats=True)["pcg_iters"]
        g.close()
    assert it[hsolver_b200.PSOLVE_MGCG] * 5 < it[hsolver_b200.PSOLVE_CG], it
