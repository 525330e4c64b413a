"""The C++ drop-in layer (include/hsolver/*.h): a driver written like the
reference's main.cpp (CYCASMesh -> DistributedMesh -> FluidSolver /
MobSolver -> Solver::solve -> result.vtk) compiles against the headers and
the in-tree library, and on the GPU writes the oracle's per-cell results,
for the reference's lid cavity and, with a ".channel" sidecar beside the
deck, for the channel physics.  The processor files the reference's
decompose step writes are read into the reference's members and checked
against the deck (on the CPU, with files written by the reference's own
code: tests/golden/proc_small)."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "hsolver_b200", "libhsolver_b200.so")


def _build(tmp_path, src="driver.cpp"):
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    exe = str(tmp_path / src.replace(".cpp", ""))
    r = subprocess.run(["sh", os.path.join(HERE, "drop_in", "build.sh"), exe, src], capture_output=True, text=True)
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


def _proc_dir(tmp_path):
    import shutil
    d = tmp_path / "run"
    shutil.copytree(os.path.join(HERE, "golden", "proc_small"), str(d))
    return str(d)


def test_processor_files_are_read_and_checked_against_the_deck(tmp_path):
    exe = _build(tmp_path, "proc_check.cpp")
    run = _proc_dir(tmp_path)
    r = subprocess.run([exe, os.path.join(HERE, "golden", "decks", "small.in")], capture_output=True, text=True,
                       cwd=run, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    got = set(r.stdout.strip().splitlines())
    # the counts the reference's decompose step wrote (meta lines of the files)
    assert {"fluid 0 cells 549", "mobs 0 cells 27", "fluid 0 faces 1881", "mobs 0 faces 108",
            "fluid 0 boundary ib_0_0 1413 45", "fluid 0 boundary wall 1458 423",
            "mobs 0 boundary ib_0_0 54 45", "mobs 0 boundary wall 99 9"} <= got
    # without processor files the deck alone is read
    r = subprocess.run([exe, os.path.join(HERE, "golden", "decks", "small.in")], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=120)
    assert r.returncode == 0 and r.stdout == "", r.stdout
    # files of another deck are refused
    r = subprocess.run([exe, os.path.join(HERE, "golden", "decks", "inner.in")], capture_output=True, text=True,
                       cwd=run, timeout=120)
    assert r.returncode == 1 and "not the deck's" in r.stdout, r.stdout


def _channel_deck(tmp_path, sidecar):
    from hsolver_b200 import cases
    deck = cases.channel(24, 12, 12, [(9, 12, 1, 4, 5, 8), (16, 19, 7, 10, 3, 6)])
    path = tmp_path / "chan.in"
    path.write_text(deck)
    (tmp_path / "chan.in.channel").write_text(sidecar)
    return str(path), deck


def test_channel_sidecar_errors_are_reported(tmp_path):
    exe = _build(tmp_path)
    path, _ = _channel_deck(tmp_path, "physics = channel\nre = 100\nviscosity = 3\n")
    r = subprocess.run([exe, path, "2", str(tmp_path / "r.vtk")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "unknown key 'viscosity'" in r.stderr, r.stderr
    (tmp_path / "chan.in.channel").write_text("re = 100\n")
    r = subprocess.run([exe, path, "2", str(tmp_path / "r.vtk")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "physics = channel" in r.stderr, r.stderr
    (tmp_path / "chan.in.channel").write_text("physics = channel\nconvection = central\n")
    r = subprocess.run([exe, path, "2", str(tmp_path / "r.vtk")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "convection must be" in r.stderr, r.stderr


@pytest.mark.gpu
def test_driver_runs_the_channel_physics_from_a_sidecar(tmp_path):
    from oracle import oracle
    exe = _build(tmp_path)
    sidecar = ("# the channel case of this deck\nphysics = channel\nre = 100\nprecision = fp64\n"
               "k_ratio = 50, 200\nq = 1.0, 2.5\np_tol = 1e-12\np_maxiter = 20000\n"
               "t_tol = 1e-12\nt_maxiter = 20000\nconvection = quick\nrichardson = 1.5\ngravity_axis = z\n")
    path, deck = _channel_deck(tmp_path, sidecar)
    vtk = str(tmp_path / "result.vtk")
    r = subprocess.run([exe, path, "3", vtk], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _read_vtk(vtk)

    o = oracle.ChannelCase(deck, re=100.0, p_tol=1e-12, p_maxiter=20000, t_tol=1e-12, t_maxiter=20000, conv=2, ri=1.5,
                           g_axis=2)
    ctype, region = oracle.OracleCase(deck).cell_types()
    o.set_solid(np.array([50.0, 200.0]), np.where(ctype == 1, np.array([1.0, 2.5])[np.maximum(region, 0)], 0.0))
    o.init()
    o.step(3)
    Nx, Ny, Nz = o.dims
    u, v, w, p, T = (o.field(f) for f in ("u", "v", "w", "p", "T"))
    exp, row = {}, 0
    for k in range(Nz):
        for j in range(Ny):
            for i in range(Nx):
                c = i + Nx * (j + Ny * k)
                if ctype[c]:
                    exp[c + 1] = (0.0, 0.0, 0.0, 0.0, T[c], -1)
                else:
                    exp[c + 1] = (p[c], u[i + (Nx + 1) * (j + Ny * k)], v[i + Nx * (j + (Ny + 1) * k)],
                                  w[i + Nx * (j + Ny * k)], T[c], row)
                    row += 1
    keys = sorted(exp)
    assert got["dims"] == (Nx, Ny, Nz)
    assert len(got["xyz"]) == len(keys)
    e = np.array([exp[k_] for k_ in keys])
    np.testing.assert_allclose(got["pressure"][:, 0], e[:, 0], rtol=1e-8, atol=1e-11)
    np.testing.assert_allclose(got["velocity"], e[:, 1:4], rtol=1e-8, atol=1e-11)
    np.testing.assert_allclose(got["temperature"][:, 0], e[:, 4], rtol=1e-8, atol=1e-11)
    assert np.array_equal(got["id"][:, 0].astype(int), e[:, 5].astype(int))
