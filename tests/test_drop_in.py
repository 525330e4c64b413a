"""The C++ drop-in layer (include/hsolver/*.h): a driver written like the
reference's main.cpp (CYCASMesh -> DistributedMesh -> FluidSolver /
MobSolver -> Solver::solve -> result.vtk) compiles against the headers and
the in-tree library, and on the GPU writes the oracle's per-cell results."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "hsolver_b200", "libhsolver_b200.so")


def _build(tmp_path):
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    exe = str(tmp_path / "driver")
    r = subprocess.run(["sh", os.path.join(HERE, "drop_in", "build.sh"), exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_driver_compiles_against_the_drop_in_headers(tmp_path):
    assert os.path.exists(_build(tmp_path))


def _read_vtk(path):
    lines = open(path).read().split("\n")
    out = {}
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("DIMENSIONS"):
            out["dims"] = tuple(int(v) for v in ln.split()[1:])
        if ln.startswith("POINTS"):
            n = int(ln.split()[1])
            out["xyz"] = np.array([[float(v) for v in lines[i + 1 + q].split()] for q in range(n)]).reshape(n, 3)
            i += n
        if ln.startswith("SCALARS") or ln.startswith("VECTORS"):
            name = ln.split()[1]
            skip = 2 if ln.startswith("SCALARS") else 1
            n = len(out["xyz"])
            out[name] = np.array([[float(v) for v in lines[i + skip + q].split()] for q in range(n)])
            i += n
        i += 1
    return out


@pytest.mark.gpu
def test_driver_writes_the_oracle_results(tmp_path):
    from oracle import oracle
    exe = _build(tmp_path)
    deck_path = os.path.join(HERE, "golden", "decks", "small.in")
    vtk = str(tmp_path / "result.vtk")
    r = subprocess.run([exe, deck_path, "3", vtk], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _read_vtk(vtk)

    deck = open(deck_path).read()
    o = oracle.OracleCase(deck)
    o.init()
    o.step(3)
    Nx, Ny, Nz = o.dims
    cx, cy, cz, fx, fy, fz, ox, oy, oz = o.meta
    ux, uy, uz = o.field("ux"), o.field("uy"), o.field("uz")
    p, t, ids, empty = o.field("p"), o.field("t"), o.row_ids(), o.fluid_empty()
    ctype, region = o.cell_types()
    exp = {}
    for k in range(cz):
        for j in range(cy):
            for i in range(cx):
                c = i + cx * (j + cy * k)
                if empty[c]:
                    continue
                g = (ox - 1 + i) + Nx * ((oy - 1 + j) + Ny * (oz - 1 + k)) + 1
                exp[g] = (p[c], ux[i + fx * (j + cy * k)], uy[i + cx * (j + fy * k)], uz[i + cx * (j + cy * k)], t[c],
                          ids[c])
    for rr in range(o.nsolid):
        m = o.solid_meta(rr)
        ts = o.solid(rr, "t")
        for k in range(m[2]):
            for j in range(m[1]):
                for i in range(m[0]):
                    gc = (m[6] - 1 + i) + Nx * ((m[7] - 1 + j) + Ny * (m[8] - 1 + k))
                    if ctype[gc] == 1 and region[gc] == rr:
                        exp[gc + 1] = (0.0, 0.0, 0.0, 0.0, ts[i + m[0] * (j + m[1] * k)], -1)
    keys = sorted(exp)
    assert got["dims"] == (Nx, Ny, Nz)
    assert len(got["xyz"]) == len(keys)
    e = np.array([exp[k_] for k_ in keys])
    np.testing.assert_allclose(got["pressure"][:, 0], e[:, 0], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(got["velocity"], e[:, 1:4], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(got["temperature"][:, 0], e[:, 4], rtol=1e-9, atol=1e-9)
    assert np.array_equal(got["id"][:, 0].astype(int), e[:, 5].astype(int))
