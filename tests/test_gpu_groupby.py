"""GroupBy on the GPU (ibfs_groupby_device, ibfs_opts.groupby = 2) against
the reference's own GroupBy order (golden fixtures recorded from
GroupBy.cuh through oracle/_ref) and the host restatement, and whole runs
with the device GroupBy against runs with the host one."""
import os

import numpy as np
import pytest

import ibfs_b200 as ib

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _device_groupby(g, src):
    import torch

    s = torch.from_numpy(np.ascontiguousarray(src, np.int32)).cuda()
    out = torch.full_like(s, -7)
    pos = torch.full_like(s, -7)
    g.groupby_device(s.data_ptr(), len(src), out.data_ptr(), pos.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), pos.cpu().numpy()


@pytest.mark.parametrize("name", ["rmat_s10", "rmat_s12", "grid_32x32", "chunglu_3k",
                                  "edge_cases"])
def test_device_groupby_matches_reference(name):
    f = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g = ib.Graph.from_csr(f["beg"], f["col"])
    try:
        out, pos = _device_groupby(g, f["src"])
        assert np.array_equal(out, f["ref_groupby"])
        assert np.array_equal(f["src"][pos], out)
    finally:
        g.close()


@pytest.mark.parametrize("n", [1, 100, 4096, 4097, 20000])
def test_device_groupby_matches_host(n):
    beg, col = ib.gen_rmat(13, 16, seed=3)
    g = ib.Graph.from_csr(beg, col)
    try:
        rng = np.random.default_rng(n)
        src = rng.integers(0, len(beg) - 1, n).astype(np.int32)  # duplicates, isolated ids
        out, pos = _device_groupby(g, src)
        assert np.array_equal(out, ib.groupby_csr(beg, col, src))
        assert np.array_equal(src[pos], out)
        # positions of equal ids stay in input order (stable)
        assert sorted(pos.tolist()) == list(range(n))
    finally:
        g.close()


@pytest.mark.parametrize("mode", [ib.MODE_PLAIN, ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP])
@pytest.mark.parametrize("layout", [ib.LAYOUT_SOURCE_MAJOR, ib.LAYOUT_VERTEX_MAJOR])
def test_run_with_device_groupby(mode, layout):
    beg, col = ib.gen_rmat(12, 16, seed=5)
    g = ib.Graph.from_csr(beg, col)
    try:
        src = ib.sample_sources(beg, col, 300, seed=6)
        a = g.run(src, width=128, mode=mode, layout=layout, groupby=1)
        b = g.run(src, width=128, mode=mode, layout=layout, groupby=2)
        assert np.array_equal(a.depth, b.depth)
        assert a.stats["traversed_edges"] == b.stats["traversed_edges"]
        # and the persistent graph replay path reuses the device regroup
        if mode == ib.MODE_PERSISTENT:
            c = g.run(src[::-1].copy(), width=128, mode=mode, layout=ib.LAYOUT_SOURCE_MAJOR,
                      groupby=2, use_graph=1)
            d = g.run(src[::-1].copy(), width=128, mode=mode, layout=ib.LAYOUT_SOURCE_MAJOR,
                      groupby=1)
            assert np.array_equal(c.depth, d.depth)
    finally:
        g.close()


def test_largest_hub_variant_same_depths():
    """groupby = 3 only changes which sources share a batch: every source's
    depths and the edge count are those of the reference GroupBy run."""
    beg, col = ib.gen_rmat(12, 16, seed=8)
    g = ib.Graph.from_csr(beg, col)
    try:
        src = ib.sample_sources(beg, col, 400, seed=9)
        a = g.run(src, width=128, groupby=1)
        b = g.run(src, width=128, groupby=3)
        assert np.array_equal(a.depth, b.depth)
        assert a.stats["traversed_edges"] == b.stats["traversed_edges"]
    finally:
        g.close()
