"""The allocation-free entry point, ibfs_run_static_scratch.

It exists for callers that cannot call cudaMalloc: a plug-in inside a
process whose own allocator owns the device memory, a latency-critical path
that may not stall in an allocation, a deployment that forbids allocation
after start-up.  Its scratch lives in a fixed device array inside the
library, so these checks make sure that array is used correctly: calls in a
row (later ones smaller, so stale contents of an earlier one would show), at
every status width, must give exactly the depths of the allocating entry
point ibfs_run and of the CPU oracle, and oversize requests must be refused
with IBFS_ERR_RANGE rather than run.

This file is collected last on purpose (test_zz_*): it must pass both alone
in a fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import ibfs_b200 as ib
from ibfs_b200 import api

pytestmark = pytest.mark.gpu


def _static_run(beg_d, col_d, V, E, src_d, n, width, out_d, stream):
    edges = C.c_int64(-1)
    st = api._lib().ibfs_run_static_scratch(
        C.c_void_p(beg_d.data_ptr()), C.c_void_p(col_d.data_ptr()), V, E,
        C.c_void_p(src_d.data_ptr()), n, width, C.c_void_p(out_d.data_ptr()),
        C.c_void_p(stream), C.byref(edges))
    return st, edges.value


def _source_major(flat: np.ndarray, n: int, V: int, width: int) -> np.ndarray:
    """Vertex-major batches (batch b at b*V*width, rows of nb bytes) to [n][V]."""
    rows = []
    for b0 in range(0, n, width):
        nb = min(width, n - b0)
        rows.append(flat[b0 * V:b0 * V + V * nb].reshape(V, nb).T)
    return np.concatenate(rows, axis=0)


def test_static_scratch_matches_ibfs_run_and_oracle():
    import torch

    import oracle

    beg, col = ib.gen_rmat(13, 16, seed=31)
    V, E = len(beg) - 1, len(col)
    dev = torch.device("cuda", 0)
    beg_d = torch.from_numpy(beg).to(dev)
    col_d = torch.from_numpy(col).to(dev)
    g = ib.Graph.from_csr(beg, col)
    stream = torch.cuda.current_stream(dev).cuda_stream
    try:
        # calls in a row, each smaller than or different from the last, so that
        # stale scratch contents of an earlier call would show; every width
        calls = [(300, 128, 1), (70, 64, 2), (500, 256, 3), (45, 32, 4)]
        for call, (n, width, seed) in enumerate(calls):
            src = ib.sample_sources(beg, col, n, seed=seed)
            src_d = torch.from_numpy(src).to(dev)
            out_static = torch.full((n * V,), 7, dtype=torch.uint8, device=dev)
            out_ref = torch.full((n * V,), 9, dtype=torch.uint8, device=dev)
            st, edges = _static_run(beg_d, col_d, V, E, src_d, n, width, out_static, stream)
            assert st == 0, f"call {call}: {api._lib().ibfs_strerror(st)}"
            res = g.run(src, width=width, concurrent=width, depth_bytes=1,
                        layout=ib.LAYOUT_VERTEX_MAJOR, on_device=True,
                        out_ptr=out_ref.data_ptr())
            torch.cuda.synchronize()
            a, b = out_static.cpu().numpy(), out_ref.cpu().numpy()
            assert np.array_equal(a, b), f"call {call}: {int((a != b).sum())} bytes differ"
            assert edges == res.stats["traversed_edges"]
            # and directly against the CPU oracle
            ref, _ = oracle.bfs(beg, col, src, 1)
            got = _source_major(a, n, V, width)
            assert np.array_equal(got, ref), f"call {call}: differs from the oracle"
            assert edges == oracle.teps(beg, ref)
    finally:
        g.close()


def test_static_scratch_refuses_oversize():
    import torch

    dev = torch.device("cuda", 0)
    # a path of 4M vertices needs more scratch than the fixed array holds
    V = 4 << 20
    beg = np.zeros(V + 1, np.int64)
    beg_d = torch.from_numpy(beg).to(dev)
    col_d = torch.zeros(1, dtype=torch.int32, device=dev)
    src_d = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.empty(V, dtype=torch.uint8, device=dev)
    st, _ = _static_run(beg_d, col_d, V, 0, src_d, 1, 32, out, 0)
    assert st == 3
    # more sources than 16 batches
    beg_s = torch.zeros(9, dtype=torch.int64, device=dev)
    src_s = torch.zeros(17 * 32, dtype=torch.int32, device=dev)
    out_s = torch.empty(17 * 32 * 8, dtype=torch.uint8, device=dev)
    st, _ = _static_run(beg_s, col_d, 8, 0, src_s, 17 * 32, 32, out_s, 0)
    assert st == 3
