"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Integer work, so the bar is bit-exact depths for every source and an exact
traversed-edge count.  Covers every status width, all three schedules, both output
layouts, partial and multiple batches, several concurrent groups, GroupBy,
the fixed and the alpha/beta direction switch, one- and two-byte depths, and
the edge cases of the reference's inputs (isolated and duplicated sources,
disconnected graphs, hubs, a long path).
"""
import numpy as np
import pytest

import ibfs_b200 as ib
import oracle

pytestmark = pytest.mark.gpu

WIDTHS = [32, 64, 128, 256]
MODES = [ib.MODE_PLAIN, ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP]


def _graph(kind: str):
    if kind == "rmat10":
        return ib.gen_rmat(10, 16, seed=11)
    if kind == "rmat13":
        return ib.gen_rmat(13, 16, seed=1)
    if kind == "rmat15":
        return ib.gen_rmat(15, 16, seed=2)
    if kind == "grid":
        return ib.gen_grid(64, 80, 0.05, 0.001, seed=4)
    if kind == "chunglu":
        return ib.gen_chung_lu(20000, 600000, 2.1, 3000.0, seed=5)
    raise KeyError(kind)


_CACHE = {}


def graph(kind):
    if kind not in _CACHE:
        beg, col = _graph(kind)
        _CACHE[kind] = (beg, col, ib.Graph.from_csr(beg, col))
    return _CACHE[kind]


def run_and_check(beg, col, g, src, layout=ib.LAYOUT_SOURCE_MAJOR, **kw):
    res = g.run(src, layout=layout, **kw)
    ref, _ = oracle.bfs_auto(beg, col, src)
    got = res.depth
    if layout == ib.LAYOUT_VERTEX_MAJOR:
        C = kw.get("concurrent", 0) or kw.get("width", 128)
        V = len(beg) - 1
        order = g.groupby(src) if kw.get("groupby") else np.asarray(src, np.int32)
        ref_o, _ = oracle.bfs_auto(beg, col, order)
        parts = []
        flat = got.reshape(-1)
        for b0 in range(0, len(src), C):
            nb = min(C, len(src) - b0)
            blk = flat[b0 * V:(b0 + nb) * V].reshape(V, nb)
            parts.append(blk.T)
        got = np.concatenate(parts, axis=0)
        ref = ref_o
    assert got.dtype == ref.dtype, (got.dtype, ref.dtype)
    assert got.shape == ref.shape
    mism = np.argwhere(got != ref)
    assert len(mism) == 0, f"{len(mism)} mismatches, first {mism[:5].tolist()}"
    assert res.stats["traversed_edges"] == oracle.teps(beg, ref)
    return res


@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("mode", MODES)
def test_rmat_widths_modes(width, mode):
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, width, seed=1)
    run_and_check(beg, col, g, src, width=width, mode=mode)


@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("mode", [ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP])
def test_partial_and_multi_batch(width, mode):
    beg, col, g = graph("rmat10")
    src = ib.sample_sources(beg, col, 2 * width + 7, seed=3)
    run_and_check(beg, col, g, src, width=width, mode=mode)
    run_and_check(beg, col, g, src[:5], width=width, mode=mode)


@pytest.mark.parametrize("groups", [1, 2, 3, 5])
@pytest.mark.parametrize("mode", [ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP])
def test_groups(groups, mode):
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 5 * 64, seed=7)
    run_and_check(beg, col, g, src, width=64, mode=mode, groups=groups)


@pytest.mark.parametrize("layout", [ib.LAYOUT_SOURCE_MAJOR, ib.LAYOUT_VERTEX_MAJOR])
@pytest.mark.parametrize("mode", MODES)
def test_layouts(layout, mode):
    beg, col, g = graph("rmat10")
    src = ib.sample_sources(beg, col, 300, seed=5)
    run_and_check(beg, col, g, src, layout=layout, width=128, mode=mode)
    run_and_check(beg, col, g, src, layout=layout, width=128, mode=mode, groupby=1)


@pytest.mark.parametrize("kind", ["grid", "chunglu", "rmat15"])
def test_graph_families(kind):
    beg, col, g = graph(kind)
    src = ib.sample_sources(beg, col, 256, seed=9)
    run_and_check(beg, col, g, src, width=128, mode=ib.MODE_PERSISTENT)
    run_and_check(beg, col, g, src[:128], width=256, mode=ib.MODE_PLAIN)
    run_and_check(beg, col, g, src, width=64, mode=ib.MODE_DEVICE_LOOP, groups=2)


@pytest.mark.parametrize("sw", [0, 1, 2, 5, 1000])
@pytest.mark.parametrize("mode", [ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP])
def test_fixed_switch_level(sw, mode):
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 128, seed=2)
    res = run_and_check(beg, col, g, src, width=128, switch_level=sw, levels_cap=64, mode=mode)
    dirs = [r["dir"] for r in res.levels if r["level"] > 0 and r["dir"] != 2]
    for r in res.levels:
        if r["level"] > 0 and r["dir"] != 2:  # dir 2: the batch's output pass
            assert r["dir"] == (0 if r["level"] <= sw else 1)
    assert dirs


@pytest.mark.parametrize("alpha,beta", [(1e-6, 1e6), (1e9, 1e-9), (14.0, 24.0), (2.0, 100.0)])
def test_alpha_beta(alpha, beta):
    beg, col, g = graph("chunglu")
    src = ib.sample_sources(beg, col, 200, seed=4)
    run_and_check(beg, col, g, src, width=256, alpha=alpha, beta=beta)


@pytest.mark.parametrize("thr", [(1, 1), (32, 512), (4, 64), (64, 64), (1000000, 1000000)])
def test_degree_thresholds(thr):
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 128, seed=8)
    run_and_check(beg, col, g, src, width=128, sml_shed=thr[0], lrg_shed=thr[1],
                  switch_level=1000)


@pytest.mark.parametrize("but", [1, 8, 1000])
def test_bottom_up_thread_limit(but):
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 200, seed=10)
    for mode in (ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP):
        run_and_check(beg, col, g, src, width=128, mode=mode, bu_thread_max=but)


def test_edge_case_graph():
    # two components, an isolated vertex, a hub, a self loop and duplicates in
    # the edge list (cleaned by the CSR builder), a 3-vertex path
    e = [(0, 1), (1, 2), (2, 3), (3, 0), (0, 0), (0, 1), (4, 5), (5, 6)]
    e += [(7, i) for i in range(8, 40)]
    u = np.array([a for a, _ in e], np.int32)
    v = np.array([b for _, b in e], np.int32)
    beg, col = ib.csr_from_edges(u, v, 41)  # vertex 40 isolated
    g = ib.Graph.from_csr(beg, col)
    src = np.array([0, 40, 4, 7, 7, 39, 2, 0], np.int32)  # isolated + duplicates
    for w in WIDTHS:
        for mode in MODES:
            run_and_check(beg, col, g, src, width=w, mode=mode)
    g.close()


def test_long_path_uint16_widening():
    n = 700
    u = np.arange(n - 1, dtype=np.int32)
    beg, col = ib.csr_from_edges(u, u + 1, n)
    g = ib.Graph.from_csr(beg, col)
    src = np.array([0, n - 1, n // 2], np.int32)
    for mode in MODES:
        res = run_and_check(beg, col, g, src, width=32, mode=mode)
        assert res.depth.dtype == np.uint16
        assert res.stats["max_level"] == n - 1
        # explicit one-byte depth must refuse instead of wrapping (comm.h:43)
        with pytest.raises(ib.IbfsError) as ei:
            g.run(src, width=32, mode=mode, depth_bytes=1)
        assert ei.value.status == 3
    g.close()


def test_graph_replay_and_stream():
    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 256, seed=12)
    ref, _ = oracle.bfs(beg, col, src)
    import torch

    out = torch.empty((len(src), len(beg) - 1), dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    try:
        for it in range(3):
            out.fill_(7)
            res = g.run(src, width=128, use_graph=1, mode=ib.MODE_PERSISTENT, on_device=True,
                        out_ptr=out.data_ptr())
            s.synchronize()
            assert np.array_equal(out.cpu().numpy(), ref)
            if it > 0:
                assert res.stats["gpu_launches"] == 1
    finally:
        g.set_stream(None)


def test_device_output_vertex_major():
    import torch

    beg, col, g = graph("rmat10")
    src = ib.sample_sources(beg, col, 100, seed=13)
    V = len(beg) - 1
    out = torch.empty(len(src) * V, dtype=torch.uint8, device="cuda")
    g.run(src, width=128, layout=ib.LAYOUT_VERTEX_MAJOR, on_device=True, out_ptr=out.data_ptr())
    got = out.cpu().numpy().reshape(V, len(src)).T
    ref, _ = oracle.bfs(beg, col, src)
    assert np.array_equal(got, ref)


def test_barrier_timeout_is_reported():
    """A withheld grid-barrier arrival makes every bounded wait run out; the
    run returns IBFS_ERR_TIMEOUT and the context stays usable."""
    beg, col, g = graph("rmat10")
    src = ib.sample_sources(beg, col, 64, seed=1)
    with pytest.raises(ib.IbfsError) as ei:
        g.run(src, width=64, mode=ib.MODE_PERSISTENT, debug_withhold=1, timeout_ms=200)
    assert ei.value.status == 6
    run_and_check(beg, col, g, src, width=64, mode=ib.MODE_PERSISTENT)


def test_bytes_alg_matches_oracle():
    import torch

    beg, col, g = graph("rmat10")
    src = ib.sample_sources(beg, col, 64, seed=21)
    ref, _ = oracle.bfs(beg, col, src)
    dev = torch.from_numpy(ref).cuda()
    for w in (64, 128):
        assert g.bytes_alg(dev.data_ptr(), len(src), 1, w) == oracle.bytes_alg(beg, col, ref, w)


def test_device_loop_replay_and_records():
    """The device-driven graph is built once and replayed; its level records
    carry the same frontiers as the persistent kernel's."""
    import torch

    beg, col, g = graph("rmat13")
    src = ib.sample_sources(beg, col, 256, seed=14)
    ref, _ = oracle.bfs(beg, col, src)
    out = torch.empty((len(src), len(beg) - 1), dtype=torch.uint8, device="cuda")
    recs = {}
    for mode in (ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP):
        for it in range(2):
            out.fill_(7)
            res = g.run(src, width=128, mode=mode, on_device=True, out_ptr=out.data_ptr(),
                        levels_cap=256)
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), ref)
        recs[mode] = [(r["batch"], r["level"], r["dir"], r["frontier"], r["frontier_edges"])
                      for r in res.levels]
        if mode == ib.MODE_DEVICE_LOOP:
            st = res.stats
            assert st["gpu_launches"] == (st["groups"] + 6 * st["n_batches"]
                                          + 4 * (st["td_levels"] + st["bu_levels"]))
    assert recs[ib.MODE_PERSISTENT] == recs[ib.MODE_DEVICE_LOOP]


def test_internal_vertex_order():
    """The device CSR is the caller's graph renamed by degree (highest first,
    ties by id) with ascending lists; results stay in caller ids."""
    import torch

    beg, col, g = graph("rmat10")
    V = len(beg) - 1
    bp, cp = g.device_csr()
    mp = g.vertex_order()
    dbeg = torch.empty(V + 1, dtype=torch.int64, device="cuda")
    dcol = torch.empty(len(col), dtype=torch.int32, device="cuda")
    dmap = torch.empty(V, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    from cuda.bindings import runtime as rt

    for dst, src_ptr, nbytes in ((dbeg, bp, 8 * (V + 1)), (dcol, cp, 4 * len(col)),
                                 (dmap, mp, 4 * V)):
        err, = rt.cudaMemcpy(dst.data_ptr(), src_ptr, nbytes,
                             rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
        assert err == rt.cudaError_t.cudaSuccess
    torch.cuda.synchronize()
    nb, nc, nm = dbeg.cpu().numpy(), dcol.cpu().numpy(), dmap.cpu().numpy()
    deg = np.diff(beg)
    order = np.argsort(-deg, kind="stable")
    assert np.array_equal(nm[order], np.arange(V))
    for new in range(0, V, 37):
        old = order[new]
        assert np.array_equal(nc[nb[new]:nb[new + 1]], np.sort(nm[col[beg[old]:beg[old + 1]]]))


@pytest.mark.parametrize("bu_filter", [0, 1, -1])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["rmat13", "grid", "chunglu"])
def test_bottom_up_frontier_filter(kind, mode, bu_filter):
    """The frontier filter (skip neighbours outside the previous frontier)
    is exact: off, on every bottom-up level, and per level (the default)."""
    beg, col, g = graph(kind)
    src = ib.sample_sources(beg, col, 128, seed=7)
    run_and_check(beg, col, g, src, width=128, mode=mode, switch_level=1, bu_filter=bu_filter)


@pytest.mark.parametrize("thresholds", [(32, 512), (1, 1)])
@pytest.mark.parametrize("mode", [ib.MODE_PLAIN, ib.MODE_DEVICE_LOOP])
@pytest.mark.parametrize("kind", ["rmat13", "chunglu"])
def test_top_down_staged_chunks(kind, mode, thresholds):
    """Large vertices' adjacency chunks staged in shared memory by bulk
    copies give the same depths; thresholds (1, 1) send every frontier
    vertex through the chunked path."""
    beg, col, g = graph(kind)
    src = ib.sample_sources(beg, col, 128, seed=9)
    run_and_check(beg, col, g, src, width=128, mode=mode, switch_level=2, td_stage=1,
                  sml_shed=thresholds[0], lrg_shed=thresholds[1])


@pytest.mark.parametrize("sparse_push", [0, 256, 4, 1])
@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("kind", ["rmat13", "rmat15", "grid", "chunglu"])
def test_sparse_source_push(kind, width, sparse_push):
    """Bottom-up levels of the device loop may hand sources with small
    frontiers to a top-down push (exit masks without their bits): depths
    and edge counts match the oracle whether the rule is off (0), selective
    (256), or pushes many sources (4, and 1: every source below the average
    frontier)."""
    beg, col, g = graph(kind)
    src = ib.sample_sources(beg, col, 2 * width + 5, seed=13)
    run_and_check(beg, col, g, src, width=width, mode=ib.MODE_DEVICE_LOOP, switch_level=1,
                  sparse_push=sparse_push)
    res = run_and_check(beg, col, g, src, width=width, mode=ib.MODE_DEVICE_LOOP, groups=2,
                        sparse_push=sparse_push)
    # with the rule on, every bottom-up level also runs the count, decision,
    # push-queue, push-chunk and bitmap-clear nodes
    st = res.stats
    per_bu = 9 if sparse_push > 0 else 4
    assert st["gpu_launches"] == (st["groups"] + 6 * st["n_batches"] + 4 * st["td_levels"]
                                  + per_bu * st["bu_levels"])


@pytest.mark.parametrize("groups", [1, 2])
def test_edgeless_sources_across_batches(groups):
    """Edgeless vertices sit at the end of the internal degree order and are
    skipped by the bottom-up sweeps; the device loop then zeroes only the
    rest of the status buffers per batch and clears each batch's edgeless
    sources itself.  Many batches in one group, most sources edgeless, two
    runs in a row: every depth must still be exact."""
    beg0, col0 = ib.gen_rmat(12, 8, seed=21)
    deg = np.diff(beg0)
    iso = np.nonzero(deg == 0)[0].astype(np.int32)
    assert len(iso) > 200
    g = ib.Graph.from_csr(beg0, col0)
    try:
        nz = ib.sample_sources(beg0, col0, 60, seed=22)
        rng = np.random.default_rng(23)
        src = np.concatenate([iso[rng.integers(0, len(iso), 200)], nz]).astype(np.int32)
        rng.shuffle(src)
        for _ in range(2):
            run_and_check(beg0, col0, g, src, width=32, mode=ib.MODE_DEVICE_LOOP, groups=groups,
                          switch_level=1)
            run_and_check(beg0, col0, g, src[:37], width=32, mode=ib.MODE_DEVICE_LOOP,
                          groups=groups, switch_level=1)
    finally:
        g.close()


@pytest.mark.parametrize("mode", MODES)
def test_directed_sinks_reached(mode):
    """A directed CSR whose second half has no out-edges but is pointed to:
    those sinks sit in the edgeless suffix of the degree order yet are
    reached at depths above 0, so neither the output pass nor the per-batch
    zeroing may treat that suffix as source-only.  Top-down only (a directed
    BFS; the bottom-up step reads the same lists as in-edges, which holds for
    symmetric graphs alone)."""
    rng = np.random.default_rng(31)
    V, H = 3000, 1500
    lists = []
    for v in range(V):
        if v >= H:
            lists.append(np.zeros(0, np.int32))
            continue
        nb = np.unique(rng.integers(0, V, 6 + (v % 11)).astype(np.int32))
        lists.append(nb[nb != v])
    beg = np.zeros(V + 1, np.int64)
    beg[1:] = np.cumsum([len(x) for x in lists])
    col = np.concatenate(lists).astype(np.int32)
    g = ib.Graph.from_csr(beg, col)
    try:
        src = np.concatenate([rng.integers(0, H, 70), rng.integers(H, V, 10)]).astype(np.int32)
        for groups in (1, 2):
            for _ in range(2):
                res = run_and_check(beg, col, g, src, width=32, mode=mode, groups=groups,
                                    switch_level=250)
                assert res.stats["bu_levels"] == 0
                assert int((res.depth[:, H:] != 0xFF).sum()) > 1000
    finally:
        g.close()
