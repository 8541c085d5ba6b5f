"""Multi-rank source sharding (ibfs_b200.shard) on CPU: two gloo ranks.

The N>1 path has no data-path collective, so what can go wrong is host
logic: the CSR replica, the GroupBy-then-contiguous-block split of
arrange_src (graph.cuh:75-95), the max-time / sum-edges reduction of
reporter (reporter.cpp:5-13) and the gather of depth rows.  Each rank here
stands a CPU graph in for its GPU replica: its ``run`` is the oracle, used
as the checker's stand-in for the device traversal, never as the product.
"""
import os
import socket

import numpy as np
import pytest

import ibfs_b200 as ib
from ibfs_b200 import shard

WORLD = 2


class _OracleGraph:
    """Test double with the Graph methods run_sharded calls."""

    def __init__(self, beg, col):
        self.beg, self.col = beg, col

    def groupby(self, src):
        return ib.groupby_csr(self.beg, self.col, src)

    def run(self, src, groupby=0, **kw):
        import oracle

        d, _ = oracle.bfs(self.beg, self.col, np.asarray(src, np.int32), 1)
        e = oracle.teps(self.beg, d)
        # a per-rank "device time" that differs between ranks, to check the max
        import torch.distributed as dist

        ms = 10.0 + 5.0 * dist.get_rank()
        return type("R", (), {"depth": d, "stats": {"device_ms": ms, "traversed_edges": e}})()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import oracle

        if rank == 0:
            beg, col = ib.gen_rmat(11, 16, seed=21)
            b, c = shard.replicate_csr(beg, col)
        else:
            b, c = shard.replicate_csr()
        ref_b, ref_c = ib.gen_rmat(11, 16, seed=21)
        assert np.array_equal(b, ref_b) and np.array_equal(c, ref_c)
        glb = ib.sample_sources(b, c, 200, seed=4)
        g = _OracleGraph(b, c)
        res = shard.run_sharded(g, glb)
        order = ib.groupby_csr(b, c, glb)
        assert np.array_equal(res.src, order[rank * 100:(rank + 1) * 100])
        assert res.job_seconds == pytest.approx(0.015)
        full = shard.gather_depths(res.depth)
        if rank == 0:
            ref, _ = oracle.bfs(b, c, order, 1)
            assert np.array_equal(full, ref)
            assert res.job_edges == oracle.teps(b, ref)
        else:
            assert full is None
        # an uneven split is refused on every rank, as the reference exits
        with pytest.raises(ib.IbfsError) as ei:
            shard.arrange_src(glb[:199], WORLD, rank)
        assert ei.value.status == 7
        open(os.path.join(out_dir, f"ok{rank}"), "w").close()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_gloo(tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_worker, args=(_free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    for r in range(WORLD):
        assert (tmp_path / f"ok{r}").exists()


def test_arrange_src_blocks():
    src = np.arange(12, dtype=np.int32)
    parts = [shard.arrange_src(src, 4, r) for r in range(4)]
    assert np.array_equal(np.concatenate(parts), src)
    assert all(len(p) == 3 for p in parts)
    with pytest.raises(ib.IbfsError):
        shard.arrange_src(src, 5, 0)
    with pytest.raises(ib.IbfsError):
        shard.arrange_src(src, 2, 2)
