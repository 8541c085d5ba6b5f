"""Serving load generator: Poisson arrivals of BFS queries against the
continuous-batching server, p50/p99 latency and aggregate GTEPS, next to the
one-query-per-launch path on the same query stream.

Both arms are measured live, in real time, on the same arrival times:

* served: a producer thread submits each query at its arrival time; waiter
  threads collect every query as soon as it is done, copying its depth rows
  into a client buffer (device memory by default: at these rates the rows,
  k x V bytes per query, exceed what PCIe can carry to the host).  Reported:
  ``latency`` = submission to depths complete in HBM (server clock) and
  ``delivered`` = submission to depths in the client's buffer.
* one query per launch: one client thread takes the queries in arrival
  order (FIFO) and runs each alone through ``ibfs_run`` (depths straight into
  a client device buffer), waiting for its arrival time when it is early.
  Latency = completion minus arrival.  When the stream outruns this path the
  queue grows without bound, so the run stops after ``budget_s``; queries not
  finished by then are counted with the latency they had reached at that
  moment (a lower bound), and the result says how many were censored.
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


def _pct(x) -> tuple[float, float]:
    x = np.asarray(x, dtype=np.float64)
    return float(np.percentile(x, 50)), float(np.percentile(x, 99))


def _warm(srv, q0: np.ndarray, batches: int, concurrent: int) -> None:
    """Untimed queries, so that the serving graph has run once before the
    measured stream starts."""
    ids = []
    left = batches * concurrent
    while left > 0:
        k = min(256, left)
        ids.append((srv.submit(np.resize(q0, k).astype(np.int32)), k))
        left -= k
    for qid, k in ids:
        srv.wait(qid, k, timeout_ms=600000, want_depth=False)


def run_served(graph, qs, arrivals, warm: bool = True, deliver: str = "device",
               waiters: int = 4, **server_kw) -> dict:
    """Replay the stream against an ibfs_server; deliver = device | host | none."""
    import torch

    import ibfs_b200 as ib

    n = len(qs)
    lat = np.zeros(n)
    dlv = np.zeros(n)
    qms = np.zeros(n)
    refused = 0
    ids: list = [None] * n
    kmax = max(len(q) for q in qs)
    V = graph.V
    bufs = []
    if deliver != "none":
        for _ in range(waiters):
            if deliver == "device":
                bufs.append(torch.empty((kmax, V), dtype=torch.uint8, device="cuda"))
            else:
                bufs.append(torch.empty((kmax, V), dtype=torch.uint8, pin_memory=True))
    with ib.Server(graph, **server_kw) as srv:
        if warm:
            C = server_kw.get("concurrent") or server_kw.get("width") or 128
            _warm(srv, qs[0], server_kw.get("round_batches", 4), C)
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

        def waiter(w):
            for i in range(w, n, waiters):
                while ids[i] is None:
                    time.sleep(0.0001)
                k = len(qs[i])
                if deliver == "none":
                    _, info = srv.wait(ids[i], k, timeout_ms=600000, want_depth=False)
                else:
                    _, info = srv.wait(ids[i], k, timeout_ms=600000,
                                       out_ptr=bufs[w].data_ptr(), on_device=deliver == "device")
                if info["status"] != 0:
                    raise RuntimeError(f"query {i} failed: {info['status']}")
                lat[i] = info["latency_ms"]
                dlv[i] = info["delivered_ms"]
                qms[i] = info["queue_ms"]

        th = [threading.Thread(target=producer)] + [threading.Thread(target=waiter, args=(w,))
                                                     for w in range(waiters)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
    edges = st["traversed_edges"] - st0["traversed_edges"]
    p50, p99 = _pct(lat)
    d50, d99 = _pct(dlv)
    return {"p50_ms": p50, "p99_ms": p99, "delivered_p50_ms": d50, "delivered_p99_ms": d99,
            "delivered_to": deliver, "mean_queue_ms": float(np.mean(qms)),
            "gteps": edges / wall / 1e9,
            "device_busy_frac": (st["busy_ms"] - st0["busy_ms"]) / 1e3 / wall,
            "batches": st["rounds"] - st0["rounds"], "launches": st["launches"] - st0["launches"],
            "queries": n, "sources": int(sum(len(q) for q in qs)), "wall_s": wall,
            "refused_retries": refused}


def run_one_per_launch(graph, qs, arrivals, width: int = 128, budget_s: float = 15.0) -> dict:
    """Each query alone (one ibfs_run per query), FIFO, live against the
    arrival times; stops after budget_s of wall time."""
    import torch

    import ibfs_b200 as ib

    V = graph.V
    kmax = max(len(q) for q in qs)
    out = torch.empty((kmax, V), dtype=torch.uint8, device="cuda")
    opts = ib.default_opts(width=width, depth_bytes=1)
    graph.run(qs[0], opts, on_device=True, out_ptr=out.data_ptr())  # warm (graph capture)
    n = len(qs)
    lat = []
    edges = 0
    t0 = time.perf_counter()
    done = 0
    for i in range(n):
        now = time.perf_counter() - t0
        if now > budget_s:
            break
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        res = graph.run(qs[i], opts, on_device=True, out_ptr=out.data_ptr())
        edges += res.stats["traversed_edges"]
        lat.append((time.perf_counter() - t0 - arrivals[i]) * 1e3)
        done += 1
    t_end = time.perf_counter() - t0
    censored = 0
    for i in range(done, n):  # not served within the budget: a lower bound
        if arrivals[i] <= t_end:
            lat.append((t_end - arrivals[i]) * 1e3)
            censored += 1
    p50, p99 = _pct(lat)
    return {"p50_ms": p50, "p99_ms": p99, "gteps": edges / t_end / 1e9, "queries_done": done,
            "queries_arrived": done + censored, "censored": censored, "wall_s": t_end,
            "latency": "arrival to depths complete in the client's device buffer"}
