"""Multi-GPU source sharding: one process per GPU over torch.distributed.

Sources are independent, so the traversal shards with no exchange on the
data path, the way the reference's MPI build does it:

* every rank holds a full replica of the CSR.  ``replicate_csr`` reads or
  generates it once on the root rank and broadcasts it (NCCL over NVLink on
  GPUs, gloo on CPU) instead of every rank reading the files;
* the global source list is put in GroupBy order (``GroupBy.cuh:6-115``,
  applied before the split at ``graph.cuh:333-339``) and cut into equal
  contiguous blocks, one per rank; an uneven split is refused
  (``arrange_src``, ``graph.cuh:75-95``, exits with "Work not even!");
* each rank traverses its block in one ``ibfs_run`` call;
* the ranks then agree on the job's time as the maximum over ranks and on
  the traversed edges as the sum (``reporter.cpp:5-13`` reduces the time
  with ``MPI_MAX``); depth rows can be gathered to one rank.

torch.distributed is only the plumbing here: the traversal itself is the
library's CUDA path, and nothing in this module computes depths.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .api import IbfsError

IBFS_ERR_INVALID_ARG = 7


def _dist():
    import torch.distributed as dist

    return dist


def _device(group=None):
    """Tensors for a collective live on the GPU under NCCL, on the host under gloo."""
    import torch

    dist = _dist()
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def arrange_src(glb_src, world: int, rank: int) -> np.ndarray:
    """This rank's contiguous block of the (GroupBy-ordered) global source list.

    Follows ``arrange_src`` (graph.cuh:75-95): the count must divide evenly by
    the number of ranks, otherwise the reference exits; here that is an
    ``IbfsError`` with status IBFS_ERR_INVALID_ARG.
    """
    glb_src = np.ascontiguousarray(glb_src, np.int32)
    if world < 1 or not 0 <= rank < world:
        raise IbfsError(IBFS_ERR_INVALID_ARG, "arrange_src: bad rank/world")
    n = len(glb_src) // world
    if n * world != len(glb_src):
        raise IbfsError(IBFS_ERR_INVALID_ARG,
                        f"arrange_src: {len(glb_src)} sources do not split evenly over {world} ranks")
    return glb_src[rank * n:(rank + 1) * n].copy()


def replicate_csr(beg=None, col=None, src_rank: int = 0, group=None):
    """Broadcast the CSR held by ``src_rank`` to every rank; returns host arrays.

    The root passes its (int64 beg, int32 col); the others pass nothing.
    Sizes go first, then the two arrays, as one broadcast each.
    """
    import torch

    dist = _dist()
    dev = _device(group)
    rank = dist.get_rank(group)
    if rank == src_rank:
        beg = np.ascontiguousarray(beg, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        sizes = torch.tensor([len(beg), len(col)], dtype=torch.int64, device=dev)
    else:
        sizes = torch.zeros(2, dtype=torch.int64, device=dev)
    dist.broadcast(sizes, src_rank, group=group)
    nb, nc = int(sizes[0]), int(sizes[1])
    if rank == src_rank:
        tb = torch.from_numpy(beg).to(dev)
        tc = torch.from_numpy(col).to(dev)
    else:
        tb = torch.empty(nb, dtype=torch.int64, device=dev)
        tc = torch.empty(nc, dtype=torch.int32, device=dev)
    dist.broadcast(tb, src_rank, group=group)
    dist.broadcast(tc, src_rank, group=group)
    return tb.cpu().numpy(), tc.cpu().numpy()


def reporter(seconds: float, edges: int, group=None) -> tuple[float, int]:
    """(max over ranks of the time, sum over ranks of the traversed edges).

    ``reporter.cpp:5-13`` takes the maximum time over ranks; the edges are
    summed so that the aggregate TEPS is edges / max time.
    """
    import torch

    dist = _dist()
    dev = _device(group)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    e = torch.tensor([int(edges)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(e, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), int(e.item())


def gather_depths(depth_local: np.ndarray, dst: int = 0, group=None):
    """Gather every rank's ``[n_local][V]`` depth rows to ``dst`` in rank order.

    Blocks are equal-sized (``arrange_src``), so rank order is the global
    source order.  Returns the ``[n][V]`` array on ``dst`` and None elsewhere.
    """
    import torch

    dist = _dist()
    dev = _device(group)
    world = dist.get_world_size(group)
    t = torch.from_numpy(np.ascontiguousarray(depth_local)).to(dev)
    if dist.get_rank(group) == dst:
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.gather(t, parts, dst=dst, group=group)
        return np.concatenate([p.cpu().numpy() for p in parts], axis=0)
    dist.gather(t, None, dst=dst, group=group)
    return None


@dataclass
class ShardResult:
    src: np.ndarray        # this rank's sources, in traversal order
    depth: np.ndarray      # [len(src)][V] depths of this rank's sources
    edges: int             # traversed edges of this rank
    seconds: float         # this rank's device time
    job_seconds: float     # max over ranks
    job_edges: int         # sum over ranks

    @property
    def job_gteps(self) -> float:
        return self.job_edges / self.job_seconds / 1e9 if self.job_seconds > 0 else 0.0


def run_sharded(graph, glb_src, group=None, groupby: bool = True, **run_kw) -> ShardResult:
    """Traverse this rank's block of ``glb_src`` on ``graph`` (a replica).

    ``graph`` is an ``ibfs_b200.Graph`` on this rank's GPU.  With ``groupby``
    the global list is GroupBy-ordered first, identically on every rank, so
    the blocks are the reference's.  Returns this rank's depths and the
    job-wide time and edge count.
    """
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    order = graph.groupby(glb_src) if groupby else np.ascontiguousarray(glb_src, np.int32)
    mine = arrange_src(order, world, rank)
    res = graph.run(mine, groupby=0, **run_kw)
    secs = res.stats["device_ms"] / 1e3
    edges = int(res.stats["traversed_edges"])
    job_s, job_e = reporter(secs, edges, group)
    return ShardResult(mine, res.depth, edges, secs, job_s, job_e)
