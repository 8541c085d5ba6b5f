"""Serving: continuous batching of BFS queries on a resident graph.

Each query's depths must be exactly its solo result whatever it was mixed
with; memory admission must hold queries back (not fail them) until rows
are free; oversize and overflowing submissions are refused."""
import threading

import numpy as np
import pytest

import ibfs_b200 as ib
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    beg, col = ib.gen_chung_lu(20000, 400000, 2.1, 2000.0, seed=5)
    g = ib.Graph.from_csr(beg, col)
    yield beg, col, g
    g.close()


def test_alone_equals_mixed(graph):
    beg, col, g = graph
    rng = np.random.default_rng(7)
    queries = []
    for i in range(24):
        k = int(np.exp(rng.uniform(0, np.log(200))))
        queries.append(ib.sample_sources(beg, col, max(1, k), seed=100 + i))
    results = {}
    with ib.Server(g, width=128, round_batches=2, max_wait_us=500) as srv:
        def client(idx):
            for i in idx:
                qid = srv.submit(queries[i])
                depth, info = srv.wait(qid, len(queries[i]))
                assert info["status"] == 0
                results[i] = depth
        ts = [threading.Thread(target=client, args=(list(range(t, 24, 4)),)) for t in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        st = srv.stats()
    assert st["completed"] == 24
    for i, q in enumerate(queries):
        solo = g.run(q, width=128).depth
        assert np.array_equal(results[i], solo), i
        ref, _ = oracle.bfs(beg, col, q)
        assert np.array_equal(results[i], ref), i


def test_memory_admission_waits_for_rows(graph):
    beg, col, g = graph
    V = len(beg) - 1
    # an arena of 100 rows; 6 queries of 60 sources each can only run one or
    # two at a time and are admitted as earlier results are collected
    with ib.Server(g, width=64, arena_bytes=100 * V, round_batches=1, max_wait_us=0) as srv:
        qs = [ib.sample_sources(beg, col, 60, seed=200 + i) for i in range(6)]
        ids = [srv.submit(q) for q in qs]
        for q, qid in zip(qs, ids):
            depth, info = srv.wait(qid, len(q))
            ref, _ = oracle.bfs(beg, col, q)
            assert np.array_equal(depth, ref)
        assert srv.stats()["arena_rows_used"] == 0


def test_refusals(graph):
    beg, col, g = graph
    V = len(beg) - 1
    with ib.Server(g, width=64, arena_bytes=50 * V, max_waiting=2, round_batches=1) as srv:
        with pytest.raises(ib.IbfsError) as ei:
            srv.submit(ib.sample_sources(beg, col, 51, seed=1))
        assert ei.value.status == 3
        big = ib.sample_sources(beg, col, 50, seed=2)
        accepted = [srv.try_submit(big) for _ in range(6)]
        assert any(a is None for a in accepted)  # the waiting queue filled up
        for qid in [a for a in accepted if a is not None]:
            depth, _ = srv.wait(qid, 50)
            assert depth.shape == (50, V)
        with pytest.raises(ib.IbfsError) as ei:
            srv.poll(123456789, 1)
        assert ei.value.status == 10


def test_batches_join_running_graph(graph):
    """Batches published while the serving graph runs are claimed by its
    groups without a new launch, and every result still equals the oracle."""
    beg, col, g = graph
    qs = [ib.sample_sources(beg, col, 128, seed=300 + i) for i in range(16)]
    with ib.Server(g, width=128, round_batches=2, max_wait_us=0) as srv:
        st0 = srv.stats()
        ids = [srv.submit(q) for q in qs]
        res = [srv.wait(qid, len(q))[0] for q, qid in zip(qs, ids)]
        st = srv.stats()
    assert st["rounds"] - st0["rounds"] == 16
    assert st["launches"] - st0["launches"] < 16 - 2, st
    for q, d in zip(qs, res):
        ref, _ = oracle.bfs(beg, col, q)
        assert np.array_equal(d, ref)


def test_late_queries_overlap_early_ones(graph):
    """A query submitted while an earlier one is still on the GPU starts
    before that one completes (its queue time is shorter than the earlier
    query's remaining latency) and both match the oracle."""
    beg, col, g = graph
    early = ib.sample_sources(beg, col, 256, seed=401)
    late = ib.sample_sources(beg, col, 8, seed=402)
    with ib.Server(g, width=32, round_batches=4, max_wait_us=0) as srv:
        qe = srv.submit(early)   # 8 batches of 32 over 4 groups
        ql = srv.submit(late)
        de, ie = srv.wait(qe, len(early))
        dl, il = srv.wait(ql, len(late))
    ref_e, _ = oracle.bfs(beg, col, early)
    ref_l, _ = oracle.bfs(beg, col, late)
    assert np.array_equal(de, ref_e) and np.array_equal(dl, ref_l)
    assert il["queue_ms"] <= ie["latency_ms"]
    assert il["delivered_ms"] >= il["latency_ms"]


def test_batch_error_stays_with_its_query():
    """One-byte depths past level 254 fail the query whose batch hit them;
    the server keeps serving and the next query is exact."""
    V_path, k = 400, 8
    edges = [(i, i + 1) for i in range(V_path - 1)]
    edges += [(V_path + a, V_path + b) for a in range(k) for b in range(a + 1, k)]
    beg, col = ib.csr_from_edges(np.array([e[0] for e in edges], np.int32),
                                 np.array([e[1] for e in edges], np.int32), V_path + k)
    g = ib.Graph.from_csr(beg, col)
    try:
        with ib.Server(g, width=32, depth_bytes=1, round_batches=1, max_wait_us=0) as srv:
            qa = srv.submit(np.array([0], np.int32))
            with pytest.raises(ib.IbfsError) as ei:
                srv.wait(qa, 1)
            assert ei.value.status == 3
            src = np.array([V_path, V_path + 3], np.int32)
            qb = srv.submit(src)
            depth, info = srv.wait(qb, 2)
            assert info["status"] == 0
            ref, _ = oracle.bfs(beg, col, src)
            assert np.array_equal(depth, ref)
    finally:
        g.close()
