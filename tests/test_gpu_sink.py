"""The depth sink: host-buffer runs stream each finished batch's rows out
while later batches traverse (replacing write_result.cuh:5-36).

Host-buffer depths must equal device-buffer depths and the CPU oracle, bit
for bit, for pinned and pageable destinations, both layouts, the device-loop
and plain schedules, and GroupBy on the host and on the GPU (whose output rows
the sink has to fetch from the device).
"""
import numpy as np
import pytest

import ibfs_b200 as ib
import oracle

pytestmark = pytest.mark.gpu

_G = {}


def graph():
    if not _G:
        beg, col = ib.gen_rmat(15, 16, seed=21)
        src = ib.sample_sources(beg, col, 1000, seed=5)  # 8 batches, 4 in flight
        ref, _ = oracle.bfs(beg, col, src, 1)
        _G.update(beg=beg, col=col, src=src, ref=ref, g=ib.Graph.from_csr(beg, col))
    return _G


def _to_source_major(flat, order, n, V, C):
    rows = {}
    for b0 in range(0, n, C):
        nb = min(C, n - b0)
        blk = flat[b0 * V:b0 * V + V * nb].reshape(V, nb)
        for j in range(nb):
            rows.setdefault(int(order[b0 + j]), []).append(blk[:, j])
    return rows


@pytest.mark.parametrize("mode", [ib.MODE_DEVICE_LOOP, ib.MODE_PLAIN])
@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("groupby", [1, 2])
def test_sink_host_equals_device_equals_oracle(mode, pinned, groupby):
    import torch

    d = graph()
    src, ref, g = d["src"], d["ref"], d["g"]
    n, V = len(src), len(d["beg"]) - 1
    if pinned:
        host = torch.full((n, V), 7, dtype=torch.uint8).pin_memory()
        out = host.numpy()
    else:
        out = np.full((n, V), 7, np.uint8)
    res = g.run(src, width=128, mode=mode, groupby=groupby, depth_bytes=1, out=out)
    assert res.depth is out or np.shares_memory(res.depth, out)
    dev = torch.full((n, V), 9, dtype=torch.uint8, device="cuda:0")
    g.run(src, width=128, mode=mode, groupby=groupby, depth_bytes=1, on_device=True,
          out_ptr=dev.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out, dev.cpu().numpy()), "host-buffer run differs from device run"
    bad = np.argwhere(out != ref)
    assert len(bad) == 0, f"{len(bad)} depth bytes differ from the oracle, first {bad[:5].tolist()}"
    assert res.stats["traversed_edges"] == oracle.teps(d["beg"], ref)


@pytest.mark.parametrize("mode", [ib.MODE_DEVICE_LOOP, ib.MODE_PLAIN])
def test_sink_vertex_major(mode):
    d = graph()
    src, g = d["src"], d["g"]
    n, V, C = len(src), len(d["beg"]) - 1, 128
    res = g.run(src, width=128, mode=mode, groupby=1, depth_bytes=1,
                layout=ib.LAYOUT_VERTEX_MAJOR)
    order = g.groupby(src)
    rows = _to_source_major(res.depth, order, n, V, C)
    for i, s in enumerate(src.tolist()):
        assert np.array_equal(rows[s].pop(0), d["ref"][i]), f"source {i}"
