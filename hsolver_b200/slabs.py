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
