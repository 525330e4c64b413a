"""Pins of the channel oracle (or_ch_*, or_cht_*) that do not go through its
own restatement: analytic solutions of the discretised physics, on the CPU.

* Series conduction.  No flow, adiabatic walls and outlet, T = Tb on the inlet
  plane, fluid | solid block | fluid along x on a random non-uniform grid, the
  heat released in the last cell plane.  All of it crosses every plane, so the
  temperature at each cell centre is Tb + (Q / A) times the sum of the thermal
  resistances between x = 0 and that centre: dx / (2k) per half cell, the two
  half cells of a fluid-solid face combined in series (the harmonic-mean face
  conductance).  The finite-volume solution reproduces this exactly, so the
  check is to round-off.
* Fully developed laminar flow in a square duct.  A block-free channel four
  heights long at Re = 10 develops within its first height; in the second half
  the axial velocity over the cross-section is the rectangular-duct series
  solution (Poiseuille flow, mean velocity u_in) and the pressure gradient is
  -dp/dx = 28.455 nu u_in / D_h^2 (f Re = 56.91 for a square duct).  The
  discretisation converges to it: from 8 x 8 to 16 x 16 cross-section
  cells the profile error falls from 3.6% to 1.0% and the pressure-gradient
  error from 5.5% to 1.5%."""
import math

import numpy as np


def test_series_conduction_through_a_block_matches_the_resistance_sum():
    from oracle import oracle
    rng = np.random.default_rng(17)
    nx = 40
    xs = np.concatenate([[0.0], np.cumsum(rng.uniform(0.02, 0.08, nx))])
    ys, zs = np.array([0.0, 0.4, 1.0]), np.array([0.0, 0.7, 1.0])
    ix = np.tile(np.arange(nx), 4)  # x index of every cell (x fastest, 2 x 2 cross-section)
    # the block fills the cross-section for cells 10 .. 29 (the solve takes the cell types directly)
    ctype = ((ix >= 10) & (ix < 30)).astype(np.uint8)
    region = np.where(ctype == 1, 0, -1).astype(np.int32)
    kf, ks, q, tb = 0.8, 37.0, 250.0, 300.0
    kcell = np.where(ctype == 1, ks, kf)
    qcell = np.where(ix == nx - 1, q, 0.0)
    zero = [np.zeros((nx + 1) * 4), np.zeros(nx * 3 * 2), np.zeros(nx * 2 * 3)]
    T = oracle.cht_solve(xs, ys, zs, ctype, region, kcell, qcell, *zero, Tb=tb, tol=1e-15, maxiter=5000, nreg=1,
                         bc=1)["T"].reshape(2, 2, nx)
    dx = np.diff(xs)
    kx = np.where((np.arange(nx) >= 10) & (np.arange(nx) < 30), ks, kf)
    flux = q * dx[-1]  # per unit cross-section area, through every plane
    res = np.empty(nx)
    res[0] = dx[0] / (2 * kx[0])
    for i in range(1, nx):
        res[i] = res[i - 1] + dx[i - 1] / (2 * kx[i - 1]) + dx[i] / (2 * kx[i])
    expect = tb + flux * res
    for j in range(2):
        for k in range(2):
            err = np.abs(T[k, j] - expect).max()
            assert err <= 1e-10 * (expect.max() - tb), (j, k, err)


def _duct_series(y, z, terms=41):
    """Axial velocity of fully developed laminar flow in the square duct
    [0,1]^2 with unit mean, at points (y, z) (the rectangular-duct series,
    summed over odd n)."""
    a = 0.5  # half side
    yy, zz = y - a, z - a
    s = np.zeros_like(yy)
    mean = 0.0
    for n in range(1, 2 * terms, 2):
        bn = n * math.pi / (2 * a)
        sign = (-1) ** ((n - 1) // 2)
        s += sign / n ** 3 * (1 - np.cosh(bn * zz) / np.cosh(bn * a)) * np.cos(bn * yy)
        # the term's cross-section mean: the y mean of cos(bn y) is sin(bn a) / (bn a) = sign / (bn a), the
        # z mean of the bracket 1 - tanh(bn a) / (bn a)
        mean += sign / n ** 3 * (sign / (bn * a)) * (1 - math.tanh(bn * a) / (bn * a))
    return s / mean


def _developed_channel(ncross):
    from hsolver_b200 import cases
    from oracle import oracle
    nx = 8 * ncross
    deck = cases.channel(nx, ncross, ncross, [], lx=4.0)
    o = oracle.ChannelCase(deck, re=10.0, p_tol=1e-10, p_maxiter=20000, t_tol=1e-2, t_maxiter=20)
    n = nx * ncross * ncross
    o.set_solid(np.zeros(0), np.zeros(n))
    o.init()
    for _ in range(3000):
        o.step(1, energy=False)
        if o.stats()["iter"] > 5 and o.stats()["global"] < 1e-7:
            break
    assert o.stats()["global"] < 1e-7
    u = o.field("u").reshape(ncross, ncross, nx + 1)
    p = o.field("p").reshape(ncross, ncross, nx)
    return u, p, nx


def _duct_errors(ncross):
    u, p, nx = _developed_channel(ncross)
    h = 1.0 / ncross
    yc = (np.arange(ncross) + 0.5) * h
    Y, Z = np.meshgrid(yc, yc, indexing="xy")  # [k, j] layout: rows z, columns y
    exact = _duct_series(Y, Z)
    # developed: the profiles at x = 2.5 and x = 3.5 agree
    f1, f2 = u[:, :, 5 * nx // 8], u[:, :, 7 * nx // 8]
    assert np.abs(f1 - f2).max() < 1e-3
    assert abs(f2.mean() - 1.0) < 1e-12  # mass conservation: the mean is u_in
    err = np.linalg.norm(f2 - exact) / np.linalg.norm(exact)
    # pressure gradient over the second half
    dpdx = (p[:, :, 7 * nx // 8].mean() - p[:, :, 5 * nx // 8].mean()) / (2 * 4.0 / 8)
    nu = 1.0 / 10.0
    return err, abs(-dpdx / (28.455 * nu) - 1.0)


def test_developed_duct_flow_converges_to_poiseuille():
    e8, g8 = _duct_errors(8)
    e16, g16 = _duct_errors(16)
    # measured: profile 3.6% / 1.0%, pressure gradient 5.5% / 1.5%
    assert e8 < 0.045 and g8 < 0.07, (e8, g8)
    assert e16 < 0.012 and g16 < 0.02, (e16, g16)
    assert e8 / e16 > 3.0 and g8 / g16 > 3.0, (e8 / e16, g8 / g16)
