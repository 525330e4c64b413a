"""Channel conjugate heat transfer (hs_channel_*) on the GPU against the CPU
oracle (oracle/hs_oracle.c, or_ch_*): the momentum sweeps bit for bit, full
outer steps with tight inner tolerances, the converged state at a global
residual of 1e-6, the mixed-precision form against FP64 (field error <= 1e-6
at the same residual, and no residual floor), mass conservation, and the
energy adjoint on the converged flow."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FACE = ["u", "v", "w"]


def _deck(nx=24, ny=12, nz=12, blocks=((9, 12, 1, 4, 5, 8),)):
    from hsolver_b200 import cases
    return cases.channel(nx, ny, nz, list(blocks))


def _pair(deck, **kw):
    import hsolver_b200
    from oracle import oracle
    g = hsolver_b200.Channel(deck, **kw)
    okw = {k: v for k, v in kw.items() if k in ("re", "pr", "u_in", "t_in", "alpha_u", "alpha_p", "alpha_t",
                                                 "mom_sweeps", "p_tol", "p_maxiter", "t_tol", "t_maxiter")}
    o = oracle.ChannelCase(deck, **okw)
    n = o.dims[0] * o.dims[1] * o.dims[2]
    ctype, region = oracle.OracleCase(deck).cell_types()
    rng = np.random.default_rng(5)
    k = rng.uniform(10.0, 1000.0, o.nreg)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, n), 0.0)
    g.set_solid(k, q)
    o.set_solid(k, q)
    g.init()
    o.init()
    return g, o, ctype


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_momentum_sweeps_bit_exact():
    g, o, _ = _pair(_deck(), re=100.0)
    for step in range(4):
        gs = g.step(1, flags=3)
        o.step(1, pressure=False, energy=False)
        for name in FACE + ["u_star", "v_star", "w_star", "d_u", "d_v", "d_w", "p"]:
            a, b = g.field(name), o.field(name)
            assert np.array_equal(a, b), (step, name, np.abs(a - b).max())
        ores = o.stats()["res"]
        for x in range(3):
            assert abs(gs["res"][x] - ores[x]) <= 1e-12 * max(ores[x], 1e-300)


@pytest.mark.parametrize("precond", [0, 1])
def test_outer_steps_match_oracle(precond):
    g, o, _ = _pair(_deck(), re=100.0, p_tol=1e-13, p_maxiter=5000, t_tol=1e-13, t_maxiter=5000, p_precond=precond)
    for step in range(5):
        gs = g.step(1)
        o.step(1)
        os_ = o.stats()
        for name in FACE + ["p", "T", "p_prime"]:
            assert _rel(g.field(name), o.field(name)) < 1e-9, (step, name)
        for x in range(5):
            assert abs(gs["res"][x] - os_["res"][x]) <= 1e-8 * max(os_["res"][x], 1e-300), (step, x)
    if precond:
        assert gs["pcg_iters"] * 4 < os_["pcg_iters"]  # the V-cycle preconditioner pays


def test_converged_state_matches_oracle_and_conserves_mass():
    deck = _deck()
    g, o, ctype = _pair(deck, re=100.0)
    ok, steps, st = g.solve_to(1e-6, 2000)
    assert ok, st
    for _ in range(steps):
        o.step(1)
    assert o.stats()["global"] <= 1e-6 * 1.5
    for name in FACE + ["p", "T"]:
        assert _rel(g.field(name), o.field(name)) < 1e-6, name
    # inflow = outflow (per unit area the faces are uniform here)
    Nx, Ny, Nz = o.dims
    u = g.field("u").reshape(Nz, Ny, Nx + 1)
    assert abs(u[:, :, 0].sum() - u[:, :, -1].sum()) <= 1e-6 * u[:, :, 0].sum()


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_steps_match_single_steps(precision):
    """hs_channel_step(n) queues its n steps back to back and applies their
    statistics afterwards (one synchronisation per 64 steps); n = 70 single
    steps and one call of 70 steps give the same fields bit for bit and the
    same statistics, normalisers included."""
    deck = _deck()
    a, _, _ = _pair(deck, re=100.0, precision=precision)
    b, _, _ = _pair(deck, re=100.0, precision=precision)
    for _ in range(70):
        sa = a.step(1)
    sb = b.step(70)
    for name in FACE + ["p", "T"]:
        assert np.array_equal(a.field(name), b.field(name)), name
    for key in ("res", "norm", "global", "iter", "pcg_iters", "t_iters", "pcg_relres", "t_relres"):
        assert sa[key] == sb[key], (key, sa[key], sb[key])


@pytest.mark.parametrize("precision", [0, 1])
def test_steps_reproducible_bit_for_bit(precision):
    """Two solvers on the 256x128x128 channel with 8 seeded blocks give the
    same fields bit for bit after 30 outer steps (reductions in a fixed
    order, no atomics, and no pass that reads what another thread of the
    same pass writes: in the mixed form the velocity correction reads u* =
    u^n + delta while it replaces u^n, so the outlet face takes its upstream
    u* from the thread of that face)."""
    import bench
    import hsolver_b200
    deck, re_, k, q, _ = bench.workload("config2")
    out = []
    for _ in range(2):
        g = hsolver_b200.Channel(deck, re=re_, precision=precision, **bench.SOLVER)
        g.set_solid(k, q)
        g.init()
        g.step(30)
        out.append({f: g.field(f) for f in FACE + ["p", "T"]})
        g.close()
    for f in FACE + ["p", "T"]:
        assert np.array_equal(out[0][f], out[1][f]), f


@pytest.mark.parametrize("precision", [0, 1])
def test_v_cycle_sweep_count_changes_only_the_path(precision):
    """The p' V-cycle's sweep count (p_mg_sweeps; the coarser levels take one
    more) is a preconditioner setting: with 1, the default (2) and 3 sweeps
    the solves take fewer CG iterations as the count grows, and the states
    converged to a global residual of 1e-8 agree to 1e-7."""
    deck = _deck(32, 16, 16, ((9, 14, 1, 6, 5, 10), (20, 24, 8, 12, 2, 6)))
    states, iters = [], []
    for sweeps in (1, 0, 3):
        g, _, _ = _pair(deck, re=100.0, precision=precision, p_mg_sweeps=sweeps)
        st = g.step(3)
        iters.append(st["pcg_iters"])
        ok, _, st = g.solve_to(1e-8, 4000)
        assert ok, (sweeps, st)
        states.append({f: g.field(f) for f in FACE + ["p", "T"]})
    assert iters[0] > iters[1] >= iters[2], iters
    for s in states[1:]:
        for name in FACE + ["T"]:
            assert _rel(s[name], states[0][name]) < 1e-7, name
        # p is defined by its differences: compare with the means removed
        a, b = s["p"] - s["p"].mean(), states[0]["p"] - states[0]["p"].mean()
        assert _rel(a, b) < 1e-7


@pytest.mark.parametrize("dims,lx,blocks", [((16, 8, 8), 2.0, ((6, 9, 1, 4, 3, 6),)),
                                             ((512, 4, 4), 64.0, ((200, 240, 1, 3, 1, 3),))])
def test_coarse_level_staging_matches_oracle(dims, lx, blocks):
    """The V-cycle levels that block 0 runs alone keep x and rhs in its shared
    memory.  16x8x8: the finest level itself is one of them (copied in from
    the CG's seeds and back for the CG); 512x4x4: the first such level
    (256x2x2, 66 KB of x and rhs in FP64) exceeds the staging area and stays
    with the grid-wide passes.  Five outer steps against the oracle with
    tight inner tolerances (T within 1e-8 on the 512-cell channel: its energy
    system is convection-dominated, and both solvers stop at a relative
    residual of 1e-13, which bounds the error of T only through the
    system's conditioning), a CG that the V-cycle shortens at least fourfold,
    and on 16x8x8 the mixed form against FP64 at a global residual of 1e-6."""
    from hsolver_b200 import cases
    deck = cases.channel(*dims, list(blocks), lx=lx)
    g, o, _ = _pair(deck, re=100.0, p_tol=1e-13, p_maxiter=5000, t_tol=1e-13, t_maxiter=5000)
    for step in range(5):
        gs = g.step(1)
        o.step(1)
        for name in FACE + ["p", "T", "p_prime"]:
            tol = 1e-8 if name == "T" and dims[0] == 512 else 1e-9
            assert _rel(g.field(name), o.field(name)) < tol, (step, name)
    assert gs["pcg_iters"] * 4 < o.stats()["pcg_iters"], (gs["pcg_iters"], o.stats()["pcg_iters"])
    if dims[0] == 16:
        g64, _, _ = _pair(deck, re=100.0)
        g32, _, _ = _pair(deck, re=100.0, precision=1)
        ok64, s64, _ = g64.solve_to(1e-6, 2000)
        ok32, s32, st = g32.solve_to(1e-6, 2000)
        assert ok64 and ok32 and s32 == s64, st
        for name in FACE + ["p", "T"]:
            assert _rel(g32.field(name), g64.field(name)) < 1e-6, name


def test_mixed_precision_against_fp64():
    deck = _deck()
    g64, _, _ = _pair(deck, re=100.0)
    g32, _, _ = _pair(deck, re=100.0, precision=1)
    ok64, s64, _ = g64.solve_to(1e-6, 2000)
    ok32, s32, st = g32.solve_to(1e-6, 2000)
    assert ok64 and ok32, st
    assert s32 == s64  # refinement: the same outer steps as the FP64 form
    for name in FACE + ["p", "T"]:
        assert _rel(g32.field(name), g64.field(name)) < 1e-6, name
    ok32, _, st = g32.solve_to(1e-9, 4000)  # no precision floor under the FP64 residual
    assert ok32 and st["global"] <= 1e-9, st


def test_adjoint_on_converged_flow_matches_oracle():
    import ctypes
    from oracle import oracle
    deck = _deck()
    g, o, ctype = _pair(deck, re=100.0)
    g.solve_to(1e-6, 2000)
    J, dq, dk, info = g.adjoint(tol=1e-12)
    oc = oracle.OracleCase(deck)
    _, region = oc.cell_types()
    grids = []
    for axis in range(3):
        a = np.empty(oc.dims[axis] + 1)
        oracle.lib().or_get_grid(oc.h, axis, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size)
        grids.append(a)
    rng = np.random.default_rng(5)
    n = ctype.size
    k = rng.uniform(10.0, 1000.0, g.nblocks)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, n), 0.0)
    kf = (1.0 * 1.0 / 100.0) / 0.71
    kcell = np.where(ctype == 1, k[np.maximum(region, 0)] * kf, kf)
    ref = oracle.cht_solve(*grids, ctype, region, kcell, q, g.field("u"), g.field("v"), g.field("w"), Tb=0.0, tol=1e-12,
                           nreg=g.nblocks, bc=1)
    assert abs(J - ref["J"]) <= 1e-10 * ref["J"]
    assert _rel(dq, ref["dJdq"]) < 1e-8
    assert _rel(dk, ref["dJdk"]) < 1e-8
    assert info["adj_iters"] <= 1.5 * info["fwd_iters"] + 5


def test_adjoint_at_config4_vs_central_differences():
    """The adjoint configuration: 128x64x64 channel, 4 seeded blocks, the
    FP64 flow converged to a global residual of 1e-6 and frozen; dJ/dq along
    16 seeded directions against central differences of the forward solve,
    relative error <= 1e-5.  The step is 1e-4 (relative to each q): with
    forward solves to 1e-13, J carries round-off noise that makes smaller
    steps noise-dominated on this grid (measured on one converged flow:
    9.6e-5 at 1e-6, 3.6e-6 at 1e-5, 2.6e-7 at 1e-4; the noise, and so the
    error at 1e-5, varies by a few times between converged flows that differ
    at the 1e-6 residual level), while the truncation error of the central
    difference of this smooth J is O(h^2).  dJ/dk per block at step 1e-3 agrees to 1e-5 of
    the largest block sensitivity (a block J hardly depends on has
    differences at the noise floor, so a relative bound would test the
    noise).  q and k are checked apart: in a joint direction the two parts
    can cancel, which measures the cancellation rather than the gradient."""
    import bench
    import hsolver_b200
    deck, re_, k, q, ctype = bench.workload("config4")
    g = hsolver_b200.Channel(deck, re=re_)
    g.set_solid(k, q)
    g.init()
    ok, steps, st = g.solve_to(1e-6, 5000)
    assert ok, st
    tol = 1e-13
    J0, dq, dk, info = g.adjoint(tol=tol, maxiter=20000)
    assert info["adj_iters"] <= 1.5 * info["fwd_iters"] + 5
    kf = (1.0 * 1.0 / re_) / 0.71          # fluid conductivity nu / Pr; k_solid = k_ratio * kf
    dk_ratio = dk * kf                      # dJ / dk_ratio
    solid = ctype == 1

    def J(kk, qq):
        g.set_solid(kk, qq)
        return g.adjoint(tol=tol, maxiter=20000)[0]

    rng = np.random.default_rng(11)
    h = 1e-4
    worst = 0.0
    for _ in range(16):
        dqd = np.where(solid, rng.standard_normal(q.size) * q, 0.0)
        fd = (J(k, q + h * dqd) - J(k, q - h * dqd)) / (2 * h)
        worst = max(worst, abs(fd - np.dot(dq, dqd)) / abs(fd))
    assert worst <= 1e-5, worst
    h = 1e-3
    scale = np.max(np.abs(dk_ratio * k))
    for b in range(k.size):
        kp, km = k.copy(), k.copy()
        kp[b] *= 1 + h
        km[b] *= 1 - h
        fd = (J(kp, q) - J(km, q)) / (2 * h)          # dJ / d(log k_b)
        assert abs(fd - dk_ratio[b] * k[b]) <= 1e-5 * scale, (b, fd, dk_ratio[b] * k[b])


@pytest.mark.parametrize("name", ["config1", "config3"])
def test_configs_match_oracle(name):
    """The configuration-1 channel and its wall-stretched variant (tanh
    clustering in y and z, cell aspect ratio up to 20): five outer steps of
    the GPU against the oracle with tight inner tolerances, and the momentum
    sweeps bit for bit with the pressure and energy solves off."""
    import bench
    import hsolver_b200
    from oracle import oracle
    deck, re_, k, q, ctype = bench.workload(name)
    kw = dict(re=re_, p_tol=1e-13, p_maxiter=5000, t_tol=1e-13, t_maxiter=5000)
    g = hsolver_b200.Channel(deck, **kw)
    o = oracle.ChannelCase(deck, **kw)
    for s_ in (g, o):
        s_.set_solid(k, q)
        s_.init()
    g.step(3, flags=3)
    o.step(3, pressure=False, energy=False)
    for f in FACE + ["u_star", "v_star", "w_star"]:
        assert np.array_equal(g.field(f), o.field(f)), f
    g.init()
    o.init()
    for _ in range(5):
        g.step(1)
        o.step(1)
    for f in FACE + ["p", "T"]:
        assert _rel(g.field(f), o.field(f)) < 1e-9, f


@pytest.mark.parametrize("precision", [0, 1])
def test_config3_converged_state_matches_oracle(precision):
    """Configuration 3 (the tanh-stretched channel, cell aspect ratio up to
    20, the mixed-precision configuration): the GPU converged to a global
    residual of 1e-6 against the oracle's converged state (tests/golden/
    channel_config3_converged.npz, made by make_channel_golden.py): the same
    number of outer steps and every field within 1e-6 relative L2."""
    import os
    import bench
    import hsolver_b200
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "channel_config3_converged.npz"))
    deck, re_, k, q, _ = bench.workload("config3")
    g = hsolver_b200.Channel(deck, re=re_, precision=precision)
    g.set_solid(k, q)
    g.init()
    ok, steps, st = g.solve_to(1e-6, 3000)
    assert ok, st
    assert steps == int(ref["steps"]), (steps, int(ref["steps"]))
    for name in FACE + ["p", "T"]:
        assert _rel(g.field(name), ref[name]) < 1e-6, name


RAGGED = {(40, 20, 12): ((9, 14, 1, 6, 4, 8), (20, 26, 10, 16, 3, 9)),
          (96, 48, 40): ((20, 30, 1, 12, 10, 20), (50, 60, 30, 40, 15, 30))}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dims", list(RAGGED))
def test_z_marching_v_cycle_matches_grid_wide(precision, dims):
    """The finest level of the p' V-cycle as z-marching passes over
    TMA-staged planes (p_level0 = 2, both colours of a sweep in one pass)
    against the grid-wide passes (p_level0 = 1, one per colour), on grids
    whose tiles are partial in x and y.  After one CG iteration p' = alpha z
    with z the V-cycle's output: z is the same bit for bit in both forms and
    alpha differs only by the summation order of its dot products, so the two
    p' fields are one scalar apart (to the rounding of the products; FP32
    storage in the mixed form)."""
    deck = _deck(*dims, blocks=RAGGED[dims])
    outs = []
    for form in (2, 1):
        g, _, _ = _pair(deck, re=100.0, precision=precision, p_maxiter=1, p_level0=form)
        st = g.step(1, flags=2)
        assert st["pcg_iters"] == 1
        outs.append(g.field("p_prime"))
        g.close()
    a, b = outs
    assert np.linalg.norm(b) > 0
    c = a.dot(b) / b.dot(b)
    tol = 1e-14 if precision == 0 else 2e-7
    assert abs(c - 1.0) < 1e-10
    assert np.linalg.norm(a - c * b) <= tol * np.linalg.norm(a)


@pytest.mark.parametrize("precision", [0, 1])
def test_z_marching_solves_match_grid_wide(precision):
    """Full p' solves to 1e-10 in both forms of the finest level: the same
    CG iteration counts (within one) and the same fields after four outer
    steps (to 1e-8)."""
    dims = (96, 48, 40)
    deck = _deck(*dims, blocks=RAGGED[dims])
    runs = []
    for form in (2, 1):
        g, _, _ = _pair(deck, re=100.0, precision=precision, p_tol=1e-10, p_level0=form)
        its = [g.step(1)["pcg_iters"] for _ in range(4)]
        runs.append((its, {f: g.field(f) for f in FACE + ["p", "T", "p_prime"]}))
        g.close()
    (ia, fa), (ib, fb) = runs
    assert all(abs(x - y) <= 1 for x, y in zip(ia, ib)), (ia, ib)
    for name in FACE + ["p", "T", "p_prime"]:
        assert _rel(fa[name], fb[name]) < 1e-8, name


def _balance_numpy(o, deck, ctype, k_ratio, q, re=100.0, pr=0.71, t_in=0.0):
    """The global balances restated from an oracle state: inlet / outlet
    volume flux, sum q V, heat leaving through the boundary (inlet
    conduction with the half-cell conductance 2 k A / dx, upwind convection
    at inlet and outlet relative to t_in)."""
    from oracle import oracle
    Nx, Ny, Nz = o.dims
    grids = []
    oc = oracle.OracleCase(deck)
    for axis in range(3):
        import ctypes
        g = np.empty(oc.dims[axis] + 1)
        oracle.lib().or_get_grid(oc.h, axis, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), g.size)
        grids.append(g)
    dx, dy, dz = (np.diff(g) for g in grids)
    A = np.outer(dz, dy)  # [k, j]
    u = o.field("u").reshape(Nz, Ny, Nx + 1)
    T = o.field("T").reshape(Nz, Ny, Nx)
    kf = 1.0 * (grids[1][-1] - grids[1][0]) / re / pr
    kcell = np.where(ctype.reshape(Nz, Ny, Nx) == 1, 0.0, kf)  # the inlet cells here are fluid
    flow_in, flow_out = (u[:, :, 0] * A).sum(), (u[:, :, -1] * A).sum()
    V = dz[:, None, None] * dy[None, :, None] * dx[None, None, :]
    src = (q.reshape(Nz, Ny, Nx) * V).sum()
    F0, F1 = -u[:, :, 0] * A, u[:, :, -1] * A
    G0 = 2.0 * kcell[:, :, 0] * A / dx[0]
    heat = (G0 * (T[:, :, 0] - t_in) + np.where(F0 > 0, F0 * T[:, :, 0], F0 * t_in)).sum()
    heat += np.where(F1 > 0, F1 * T[:, :, -1], F1 * t_in).sum()
    return np.array([flow_in, flow_out, src, heat])


@pytest.mark.parametrize("precision", [0, 1])
def test_global_balances(precision):
    """hs_channel_balance (FP64 sums on the GPU) against the same sums
    restated in NumPy on the oracle's state after the same steps, and the
    balances' closure at convergence: inflow = outflow, heat source = heat
    leaving through the boundary."""
    deck = _deck()
    kw = dict(re=100.0, p_tol=1e-13, p_maxiter=5000, t_tol=1e-13, t_maxiter=5000)
    g, o, ctype = _pair(deck, precision=precision, **kw)
    n = o.dims[0] * o.dims[1] * o.dims[2]
    rng = np.random.default_rng(5)  # _pair's block physics
    k = rng.uniform(10.0, 1000.0, o.nreg)
    q = np.where(ctype == 1, rng.uniform(0.5, 2.0, n), 0.0)
    g.step(4)
    o.step(4)
    b = g.balance()
    got = np.array([b["flow_in"], b["flow_out"], b["heat_source"], b["heat_out"]])
    exp = _balance_numpy(o, deck, ctype, k, q)
    tol = 1e-9 if precision == 0 else 1e-6
    assert np.all(np.abs(got - exp) <= tol * np.abs(exp)), (got, exp)
    ok, _, _ = g.solve_to(1e-8, 4000)
    assert ok
    b = g.balance()
    assert abs(b["flow_in"] - b["flow_out"]) <= 1e-8 * b["flow_in"], b
    assert abs(b["heat_source"] - b["heat_out"]) <= 1e-5 * b["heat_source"], b
    g.close()
