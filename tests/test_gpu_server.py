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
