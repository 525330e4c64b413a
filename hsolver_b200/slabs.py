"""z-slab sharding of the channel grid over ranks: the partition, the halo
exchange of one plane per neighbour and the global reductions.

The reference's only parallelism is domain decomposition over MPI ranks
(Scotch parts, mesh/mesh.cpp:735-1122) with a halo exchange per sweep
(fluid_solver.h:641-645, 559-563, 473-477) and a residual allreduce
(fluid_solver.h:485).  On B200 the whole mesh of every target case fits one
GPU, so the product runs replicas; a mesh beyond one GPU's 180 GB splits into
contiguous z-slabs, one per rank, each with one ghost plane below and above:

* partition: slab_bounds gives rank r the interior planes [k0, k1), sizes
  differing by at most one;
* exchange: each rank sends its first interior plane down and its last one
  up and receives its ghost planes from the neighbours (point-to-point, so
  over NCCL each plane crosses NVLink once into the receiver's own memory:
  no rank reads another rank's memory);
* reductions: dot products and residual norms are per-rank partial sums
  added by an all-reduce in FP64.

The local compute (the stencil passes over a slab with its ghost planes) is
the caller's; the arrays here are torch tensors of shape (nz_local + 2, ny,
nx) on the rank's device ("cuda" with NCCL, "cpu" with gloo)."""


def slab_bounds(nz, world, rank):
    """Interior planes [k0, k1) of `rank` among `world` contiguous slabs of
    nz planes (the first nz % world slabs one plane larger)."""
    if world < 1 or not (0 <= rank < world) or nz < world:
        raise ValueError("need 0 <= rank < world <= nz")
    base, extra = divmod(nz, world)
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def exchange_halo(t, dist, group=None):
    """Fill the ghost planes t[0] and t[-1] of this rank's slab from the
    neighbouring ranks' first and last interior planes; the ghosts of the
    end slabs are left as they are (the boundary).  Every rank takes the same
    steps in the same order: sends are posted before receives."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    reqs = []
    up, down = rank + 1 < world, rank > 0
    if down:
        reqs.append(dist.isend(t[1].contiguous(), rank - 1, group=group, tag=1))
    if up:
        reqs.append(dist.isend(t[-2].contiguous(), rank + 1, group=group, tag=2))
    recv = []
    if down:
        buf = t[0].new_empty(t[0].shape)
        reqs.append(dist.irecv(buf, rank - 1, group=group, tag=2))
        recv.append((0, buf))
    if up:
        buf = t[-1].new_empty(t[-1].shape)
        reqs.append(dist.irecv(buf, rank + 1, group=group, tag=1))
        recv.append((-1, buf))
    for r in reqs:
        r.wait()
    for idx, buf in recv:
        t[idx].copy_(buf)
    return t


def allreduce_sum(value, dist, device, group=None):
    """The FP64 sum over ranks of a per-rank partial sum."""
    import torch
    x = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)
    return float(x.item())


# ---------------------------------------------------------------- the sharded p' solve on GPUs
class SlabPCG:
    """One slab of the pressure-correction system on a GPU (hs_slab_* of the
    C ABI): face couplings gx (nz, ny, nx + 1), gy (nz, ny + 1, nx), gz
    (nz + 1, ny, nx) with gz[0] and gz[nz] the slab's bottom and top faces,
    and the right-hand side b (nz, ny, nx), numpy arrays.  coarse = (agg,
    kg0, nzg): the two-level preconditioner's global coarse grid of agg^3-cell
    aggregates, this slab starting at global plane kg0 of nzg."""

    def __init__(self, nx, ny, nz, device=0, coarse=None):
        import ctypes
        from . import load, HsError
        L = load()
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        sig = {"hs_slab_create": [ctypes.c_int] * 4 + [ctypes.POINTER(vp)],
               "hs_slab_set_system": [vp, vp, vp, vp, vp], "hs_slab_begin": [vp, dp], "hs_slab_precond": [vp, dp],
               "hs_slab_direction": [vp, ctypes.c_double, ctypes.c_int], "hs_slab_apply": [vp, dp],
               "hs_slab_update": [vp, ctypes.c_double, dp], "hs_slab_plane_size": [vp, ctypes.POINTER(ctypes.c_longlong)],
               "hs_slab_halo_get": [vp, vp, vp], "hs_slab_halo_put": [vp, vp, vp], "hs_slab_get": [vp, ctypes.c_int, vp],
               "hs_slab_set_coarse": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
               "hs_slab_coarse_sizes": [vp, ctypes.POINTER(ctypes.c_longlong)],
               "hs_slab_coarse_partial": [vp, vp, vp, vp], "hs_slab_coarse_build": [vp, vp, vp, vp],
               "hs_slab_restrict": [vp, vp], "hs_slab_coarse_correct": [vp, vp, dp]}
        for name, args in sig.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = ctypes.c_int
        L.hs_slab_destroy.argtypes = [vp]
        L.hs_slab_destroy.restype = None
        import torch
        self._L, self._ct, self._err = L, ctypes, HsError
        self.dims = (nx, ny, nz)
        self.device = device
        self.torch_device = torch.device("cuda", device)
        self.h = None
        h = vp()
        self._check(L.hs_slab_create(nx, ny, nz, device, ctypes.byref(h)))
        self.h = h
        n = ctypes.c_longlong()
        self._check(L.hs_slab_plane_size(h, ctypes.byref(n)))
        self.plane = n.value
        self.coarse = coarse
        self.coarse_ready = False
        if coarse is not None:
            agg, kg0, nzg = coarse
            self._check(L.hs_slab_set_coarse(h, int(agg), int(kg0), int(nzg)))
            n4 = (ctypes.c_longlong * 4)()
            self._check(L.hs_slab_coarse_sizes(h, n4))
            self.coarse_sizes = tuple(int(v) for v in n4)

    def _check(self, rc):
        if rc < 0:
            raise self._err(rc, self._L.hs_last_error(None).decode())

    def _scalar(self, fn, *args):
        v = self._ct.c_double()
        self._check(fn(self.h, *args, self._ct.byref(v)))
        return v.value

    def set_system(self, gx, gy, gz, b):
        import numpy as np
        nx, ny, nz = self.dims
        arrs = [np.ascontiguousarray(a, np.float64) for a in (gx, gy, gz, b)]
        for a, shape in zip(arrs, [(nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx), (nz, ny, nx)]):
            if a.shape != shape:
                raise ValueError("expected shape %s, got %s" % (shape, a.shape))
        self._check(self._L.hs_slab_set_system(self.h, *[a.ctypes.data for a in arrs]))
        self.coarse_ready = False

    def coarse_partial(self):
        """This slab's partial coarse face couplings (gx, gy, gz of the coarse grid)."""
        import numpy as np
        out = [np.zeros(n) for n in self.coarse_sizes[:3]]
        self._check(self._L.hs_slab_coarse_partial(self.h, *[a.ctypes.data for a in out]))
        return out

    def coarse_build(self, cg):
        import numpy as np
        arrs = [np.ascontiguousarray(a, np.float64) for a in cg]
        self._check(self._L.hs_slab_coarse_build(self.h, *[a.ctypes.data for a in arrs]))
        self.coarse_ready = True

    def restrict(self):
        import numpy as np
        out = np.zeros(self.coarse_sizes[3])
        self._check(self._L.hs_slab_restrict(self.h, out.ctypes.data))
        return out

    def coarse_correct(self, rc):
        import numpy as np
        a = np.ascontiguousarray(rc, np.float64)
        return self._scalar(self._L.hs_slab_coarse_correct, a.ctypes.data)

    def begin(self):
        return self._scalar(self._L.hs_slab_begin)

    def precond(self):
        return self._scalar(self._L.hs_slab_precond)

    def direction(self, beta, first):
        self._check(self._L.hs_slab_direction(self.h, float(beta), int(first)))

    def apply(self):
        return self._scalar(self._L.hs_slab_apply)

    def update(self, alpha):
        return self._scalar(self._L.hs_slab_update, float(alpha))

    def halo_get(self, lo, hi):
        """p's first and last interior planes into torch CUDA tensors (or None)."""
        self._check(self._L.hs_slab_halo_get(self.h, lo.data_ptr() if lo is not None else None,
                                             hi.data_ptr() if hi is not None else None))

    def halo_put(self, lo, hi):
        """torch CUDA tensors (or None) into p's ghost planes below and above."""
        self._check(self._L.hs_slab_halo_put(self.h, lo.data_ptr() if lo is not None else None,
                                             hi.data_ptr() if hi is not None else None))

    def field(self, which="x"):
        import numpy as np
        nx, ny, nz = self.dims
        out = np.empty((nz, ny, nx))
        self._check(self._L.hs_slab_get(self.h, {"x": 0, "r": 1, "p": 2, "s": 3}[which], out.ctypes.data))
        return out

    def close(self):
        if self.h:
            self._L.hs_slab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _exchange_local(slabs, bufs):
    """Each slab's p boundary planes into its neighbours' ghost planes, for
    consecutive slabs of one process (device-to-device copies)."""
    for a, b in zip(slabs[:-1], slabs[1:]):
        up, down = bufs
        a.halo_get(None, up)    # a's top plane -> b's lower ghost
        b.halo_get(down, None)  # b's bottom plane -> a's upper ghost
        b.halo_put(up, None)
        a.halo_put(None, down)


def _exchange_dist(slab, bufs, dist, group):
    """This rank's slab's p boundary planes to the neighbouring ranks and
    theirs into its ghost planes (the same steps as exchange_halo, over the
    process group: NCCL send/recv into the receiver's own memory)."""
    import torch
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo_send, hi_send, lo_recv, hi_recv = bufs
    down, up = rank > 0, rank + 1 < world
    slab.halo_get(lo_send if down else None, hi_send if up else None)
    reqs = []
    if down:
        reqs.append(dist.isend(lo_send, rank - 1, group=group, tag=1))
    if up:
        reqs.append(dist.isend(hi_send, rank + 1, group=group, tag=2))
    if down:
        reqs.append(dist.irecv(lo_recv, rank - 1, group=group, tag=2))
    if up:
        reqs.append(dist.irecv(hi_recv, rank + 1, group=group, tag=1))
    for r in reqs:
        r.wait()
    if lo_recv.is_cuda:  # NCCL's receives run on the current stream; the slab copies on its own
        torch.cuda.current_stream(lo_recv.device).synchronize()
    slab.halo_put(lo_recv if down else None, hi_recv if up else None)


def slab_pcg_solve(slabs, tol=1e-8, maxiter=1000, dist=None, group=None):
    """CG on the pressure-correction system sharded into z-slabs, each
    preconditioned by its own V-cycle (block Jacobi), plus, when the slabs
    carry a coarse grid, the additive global coarse correction (its
    couplings summed over the slabs once per system, the restricted residual
    summed every application).  `slabs`: SlabPCG (or
    any object with its methods, `plane` and `torch_device`): this
    process's slabs, bottom to top: every slab of the domain when dist is
    None (one process, one or more slabs on its GPU), or this rank's one slab
    with dist = torch.distributed (NCCL), ranks in z order.  Dot products are
    the slabs' FP64 partial sums, all-reduced.  Returns (iterations,
    ||r|| / ||b||)."""
    import torch
    if dist is not None and len(slabs) != 1:
        raise ValueError("one slab per rank with a process group")
    dev = slabs[0].torch_device
    plane = slabs[0].plane
    if dist is None:
        bufs = (torch.empty(plane, dtype=torch.float64, device=dev), torch.empty(plane, dtype=torch.float64, device=dev))
        exchange = lambda: _exchange_local(slabs, bufs)  # noqa: E731
    else:
        bufs = tuple(torch.empty(plane, dtype=torch.float64, device=dev) for _ in range(4))
        exchange = lambda: _exchange_dist(slabs[0], bufs, dist, group)  # noqa: E731

    def total(vals):
        s = 0.0
        for v in vals:
            s += v
        return allreduce_sum(s, dist, dev, group) if dist is not None else s

    def total_vec(vecs):
        # element-wise FP64 sum over this process's slabs and over the ranks
        out = vecs[0].copy()
        for v in vecs[1:]:
            out += v
        if dist is not None:
            t = torch.from_numpy(out).to(dev)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            out = t.cpu().numpy()
        return out

    coarse = getattr(slabs[0], "coarse", None) is not None
    if coarse and not all(s.coarse_ready for s in slabs):
        parts = [s.coarse_partial() for s in slabs]
        cg = [total_vec([p[a] for p in parts]) for a in range(3)]
        for s in slabs:
            s.coarse_build(cg)

    def precondition():
        if not coarse:
            return total([s.precond() for s in slabs])
        for s in slabs:
            s.precond()
        rc = total_vec([s.restrict() for s in slabs])
        return total([s.coarse_correct(rc) for s in slabs])

    bb = total([s.begin() for s in slabs])
    if bb == 0.0:
        return 0, 0.0
    rz = precondition()
    for s in slabs:
        s.direction(0.0, True)
    rr, it = bb, 0
    while it < maxiter and rr / bb >= tol * tol:
        it += 1
        exchange()
        sp = total([s.apply() for s in slabs])
        alpha = rz / sp
        rr = total([s.update(alpha) for s in slabs])
        if rr / bb < tol * tol or it >= maxiter:
            break
        rz_new = precondition()
        beta = rz_new / rz
        rz = rz_new
        for s in slabs:
            s.direction(beta, False)
    return it, (rr / bb) ** 0.5
