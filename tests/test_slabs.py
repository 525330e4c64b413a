"""z-slab sharding (hsolver_b200/slabs.py) on the host with gloo ranks: the
p' operator of a channel-like system (face couplings, solid cells with none,
the outlet face to p' = 0 outside) applied slab by slab after the halo
exchange equals the single-domain operator bit for bit, and a CG whose dot
products are all-reduced over the slabs converges to the single-domain CG's
solution.  2 and 3 ranks on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest

NZ, NY, NX = 11, 6, 9


def _system(seed=3):
    rng = np.random.default_rng(seed)
    solid = np.zeros((NZ, NY, NX), bool)
    solid[3:6, 1:4, 2:5] = True
    gx = rng.uniform(0.5, 2.0, (NZ, NY, NX + 1))
    gy = rng.uniform(0.5, 2.0, (NZ, NY + 1, NX))
    gz = rng.uniform(0.5, 2.0, (NZ + 1, NY, NX))
    gx[:, :, 0] = 0.0  # inlet: fixed velocity, no coupling
    gy[:, 0, :] = gy[:, -1, :] = 0.0  # walls
    gz[0] = gz[-1] = 0.0
    # no coupling through a face of a solid cell
    gx[:, :, 1:][solid] = 0.0
    gx[:, :, :-1][solid] = 0.0
    gy[:, 1:, :][solid] = 0.0
    gy[:, :-1, :][solid] = 0.0
    gz[1:][solid] = 0.0
    gz[:-1][solid] = 0.0
    b = np.where(solid, 0.0, rng.standard_normal((NZ, NY, NX)))
    return gx, gy, gz, b


def apply_slab(x, gx, gy, gz):
    """y = A x on planes 1..n of x (shape (n + 2, ny, nx), ghost planes 0 and
    n + 1), couplings of those planes (gz with n + 1 face planes); p' = 0
    beyond the outlet face gx[..., nx]."""
    xi = x[1:-1]
    d = gx[:, :, :-1] + gx[:, :, 1:] + gy[:, :-1, :] + gy[:, 1:, :] + gz[:-1] + gz[1:]
    y = d * xi
    y[:, :, 1:] -= gx[:, :, 1:-1] * xi[:, :, :-1]
    y[:, :, :-1] -= gx[:, :, 1:-1] * xi[:, :, 1:]
    y[:, 1:, :] -= gy[:, 1:-1, :] * xi[:, :-1, :]
    y[:, :-1, :] -= gy[:, 1:-1, :] * xi[:, 1:, :]
    y -= gz[:-1] * x[:-2]
    y -= gz[1:] * x[2:]
    return y


def cg(apply, b, dot, tol=1e-10, maxiter=500):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = dot(r, r)
    bb = rr
    it = 0
    while it < maxiter and rr > tol * tol * bb:
        s = apply(p)
        alpha = rr / dot(s, p)
        x += alpha * p
        r -= alpha * s
        rn = dot(r, r)
        p = r + (rn / rr) * p
        rr = rn
        it += 1
    return x, it


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from hsolver_b200 import slabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        gx, gy, gz, b = _system()
        k0, k1 = slabs.slab_bounds(NZ, world, rank)
        lgx, lgy, lgz = gx[k0:k1], gy[k0:k1], gz[k0:k1 + 1]
        rng = np.random.default_rng(11)
        xfull = rng.standard_normal((NZ, NY, NX))
        x = torch.zeros((k1 - k0 + 2, NY, NX), dtype=torch.float64)
        x[1:-1] = torch.from_numpy(xfull[k0:k1])
        slabs.exchange_halo(x, dist)
        y = apply_slab(x.numpy(), lgx, lgy, lgz)

        def app(v):
            t = torch.zeros((k1 - k0 + 2, NY, NX), dtype=torch.float64)
            t[1:-1] = torch.from_numpy(v)
            slabs.exchange_halo(t, dist)
            return apply_slab(t.numpy(), lgx, lgy, lgz)

        sol, it = cg(app, b[k0:k1], lambda u, v: slabs.allreduce_sum(float((u * v).sum()), dist, "cpu"))
        q.put((rank, k0, k1, y, sol, it))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_slab_bounds_cover_the_planes():
    from hsolver_b200 import slabs
    for nz in (8, 11, 128):
        for world in (1, 2, 3, 8):
            b = [slabs.slab_bounds(nz, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == nz
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            assert max(e - s for s, e in b) - min(e - s for s, e in b) <= 1
    with pytest.raises(ValueError):
        slabs.slab_bounds(2, 3, 0)


@pytest.mark.parametrize("world", [2, 3])
def test_slab_operator_and_cg_match_the_single_domain(world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    gx, gy, gz, b = _system()
    xfull = np.random.default_rng(11).standard_normal((NZ, NY, NX))
    pad = np.zeros((NZ + 2, NY, NX))
    pad[1:-1] = xfull
    y_ref = apply_slab(pad, gx, gy, gz)
    sol_ref, it_ref = cg(lambda v: apply_slab(np.concatenate([np.zeros((1, NY, NX)), v, np.zeros((1, NY, NX))]),
                                              gx, gy, gz), b, lambda u, v: float((u * v).sum()))
    y = np.zeros_like(y_ref)
    sol = np.zeros_like(sol_ref)
    its = set()
    for rank, k0, k1, yl, sl, it in got:
        y[k0:k1] = yl
        sol[k0:k1] = sl
        its.add(it)
    assert np.array_equal(y, y_ref)  # every cell's sum in the same order: bit for bit
    assert len(its) == 1 and abs(its.pop() - it_ref) <= 1
    assert np.linalg.norm(sol - sol_ref) <= 1e-9 * np.linalg.norm(sol_ref)


class NumpySlab:
    """The interface of hsolver_b200.slabs.SlabPCG in NumPy on the CPU
    (Jacobi in place of the V-cycle: block diagonal and SPD as well), so that
    the sharded CG driver runs over gloo ranks without a GPU."""

    def __init__(self, gx, gy, gz, b):
        import torch
        self.gx, self.gy, self.gz, self.b = gx, gy, gz, b
        nz, ny, nx = b.shape
        self.d = gx[:, :, :-1] + gx[:, :, 1:] + gy[:, :-1, :] + gy[:, 1:, :] + gz[:-1] + gz[1:]
        self.x = np.zeros((nz + 2, ny, nx))
        self.r = np.zeros((nz + 2, ny, nx))
        self.p = np.zeros((nz + 2, ny, nx))
        self.s = np.zeros((nz + 2, ny, nx))
        self.plane = ny * nx
        self.torch_device = torch.device("cpu")

    def begin(self):
        self.x[:] = 0.0
        self.r[1:-1] = self.b
        return float((self.b * self.b).sum())

    def precond(self):
        self.z = np.where(self.d > 0, self.r[1:-1] / np.where(self.d > 0, self.d, 1.0), 0.0)
        return float((self.r[1:-1] * self.z).sum())

    def direction(self, beta, first):
        self.p[1:-1] = self.z if first else self.z + beta * self.p[1:-1]

    def apply(self):
        self.s[1:-1] = apply_slab(self.p, self.gx, self.gy, self.gz)
        return float((self.s[1:-1] * self.p[1:-1]).sum())

    def update(self, alpha):
        self.x[1:-1] += alpha * self.p[1:-1]
        self.r[1:-1] -= alpha * self.s[1:-1]
        return float((self.r[1:-1] ** 2).sum())

    def halo_get(self, lo, hi):
        import torch
        if lo is not None:
            lo.copy_(torch.from_numpy(self.p[1].ravel().copy()))
        if hi is not None:
            hi.copy_(torch.from_numpy(self.p[-2].ravel().copy()))

    def halo_put(self, lo, hi):
        if lo is not None:
            self.p[0] = lo.numpy().reshape(self.p[0].shape)
        if hi is not None:
            self.p[-1] = hi.numpy().reshape(self.p[-1].shape)


def _pcg_rank(rank, world, port, q):
    import torch.distributed as dist
    from hsolver_b200 import slabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        gx, gy, gz, b = _system()
        k0, k1 = slabs.slab_bounds(NZ, world, rank)
        s = NumpySlab(gx[k0:k1], gy[k0:k1], gz[k0:k1 + 1], b[k0:k1])
        it, rel = slabs.slab_pcg_solve([s], tol=1e-10, maxiter=500, dist=dist)
        q.put((rank, k0, k1, s.x[1:-1].copy(), it, rel))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_pcg_driver_over_ranks_matches_one_process(world):
    """hsolver_b200.slabs.slab_pcg_solve with one slab per gloo rank (halo
    planes by send/recv, dots all-reduced) gives the iterates of the same
    slabs driven in one process (halo planes copied): the same iteration
    count and the solution to round-off; both solve the global system."""
    import multiprocessing as mp
    from hsolver_b200 import slabs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_pcg_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    gx, gy, gz, b = _system()
    local = []
    for r in range(world):
        k0, k1 = slabs.slab_bounds(NZ, world, r)
        local.append(NumpySlab(gx[k0:k1], gy[k0:k1], gz[k0:k1 + 1], b[k0:k1]))
    it_loc, rel_loc = slabs.slab_pcg_solve(local, tol=1e-10, maxiter=500)
    x_loc = np.concatenate([s.x[1:-1] for s in local])
    x = np.zeros_like(x_loc)
    for rank, k0, k1, xl, it, rel in got:
        x[k0:k1] = xl
        assert abs(it - it_loc) <= 1 and rel < 1e-10
    assert np.linalg.norm(x - x_loc) <= 1e-9 * np.linalg.norm(x_loc)
    pad = lambda v: np.concatenate([np.zeros((1, NY, NX)), v, np.zeros((1, NY, NX))])  # noqa: E731
    res = b - apply_slab(pad(x), gx, gy, gz)
    assert np.linalg.norm(res) <= 1e-9 * np.linalg.norm(b)
