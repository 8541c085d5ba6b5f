"""Serving load generator: Poisson arrivals of BFS queries against the
continuous-batching server, p50/p99 latency and aggregate GTEPS, next to the
one-query-per-launch path on the same query stream.

Latency is measured by the server from submission to the query's depths
being complete in device memory (results are left on the device and
collected without a host copy).  The one-query-per-launch figure runs every
query alone through ibfs_run (persistent kernel, device output), measures
its device time, and replays the same arrival times through a single FIFO
server with those service times.
"""
from __future__ import annotations

import threading
import time

import numpy as np


def query_stream(pool: np.ndarray, n_queries: int, rate: float, seed: int, max_k: int = 256):
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.floor(np.exp(rng.uniform(0.0, np.log(max_k + 1), n_queries))), 1,
                    max_k).astype(int)
    gaps = rng.exponential(1.0 / rate, n_queries)
    arrivals = np.cumsum(gaps) - gaps[0]
    qs = [pool[rng.integers(0, len(pool), k)].astype(np.int32) for k in sizes]
    return qs, arrivals


def _warm(srv, q0: np.ndarray, round_sources: int, concurrent: int) -> None:
    """Untimed rounds of 1..round_batches batches, so that the launch graphs
    of every round shape exist before the measured stream starts."""
    for total in range(concurrent, round_sources + 1, concurrent):
        ids = []
        left = total
        while left > 0:
            k = min(256, left)
            ids.append((srv.submit(np.resize(q0, k).astype(np.int32)), k))
            left -= k
        for qid, k in ids:
            srv.wait(qid, k, timeout_ms=600000, want_depth=False)


def run_served(graph, qs, arrivals, warm: bool = True, **server_kw) -> dict:
    import ibfs_b200 as ib

    lat, queue, refused = [], [], 0
    done_evt = threading.Event()
    ids: list = [None] * len(qs)
    with ib.Server(graph, **server_kw) as srv:
        if warm:
            C = server_kw.get("concurrent") or server_kw.get("width") or 128
            _warm(srv, qs[0], C * server_kw.get("round_batches", 4), C)
        st0 = srv.stats()
        t0 = time.perf_counter()

        def producer():
            nonlocal refused
            for i, (q, at) in enumerate(zip(qs, arrivals)):
                dt = at - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                while True:
                    qid = srv.try_submit(q)
                    if qid is not None:
                        ids[i] = qid
                        break
                    refused += 1
                    time.sleep(0.0005)
            done_evt.set()

        th = threading.Thread(target=producer)
        th.start()
        for i, q in enumerate(qs):
            while ids[i] is None:
                time.sleep(0.0002)
            _, info = srv.wait(ids[i], len(q), timeout_ms=600000, want_depth=False)
            if info["status"] != 0:
                raise RuntimeError(f"query {i} failed: {info['status']}")
            lat.append(info["latency_ms"])
            queue.append(info["queue_ms"])
        th.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
    lat = np.asarray(lat)
    edges = st["traversed_edges"] - st0["traversed_edges"]
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_queue_ms": float(np.mean(queue)), "gteps": edges / wall / 1e9,
            "device_busy_frac": (st["busy_ms"] - st0["busy_ms"]) / 1e3 / wall,
            "rounds": st["rounds"] - st0["rounds"],
            "queries": len(qs), "sources": int(sum(len(q) for q in qs)), "wall_s": wall,
            "refused_retries": refused}


def run_one_per_launch(graph, qs, arrivals, width: int = 128) -> dict:
    """Each query alone (one launch per query), FIFO single server replay."""
    import torch

    import ibfs_b200 as ib

    V = graph.V
    out = torch.empty((256, V), dtype=torch.uint8, device="cuda")
    opts = ib.default_opts(width=width, depth_bytes=1)
    svc, edges = [], 0
    for q in qs:
        res = graph.run(q, opts, on_device=True, out_ptr=out.data_ptr())
        svc.append(res.stats["device_ms"] / 1e3)
        edges += res.stats["traversed_edges"]
    t_free, lat = 0.0, []
    for at, s in zip(arrivals, svc):
        start = max(at, t_free)
        t_free = start + s
        lat.append((t_free - at) * 1e3)
    span = max(t_free, arrivals[-1]) - arrivals[0]
    lat = np.asarray(lat)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "gteps": edges / span / 1e9, "service_ms_mean": float(np.mean(svc) * 1e3)}
