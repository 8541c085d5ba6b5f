"""The per-graph autotuner returns options that are valid and at least as
fast as its starting point on the sample it timed; results stay exact."""
import numpy as np
import pytest

import ibfs_b200 as ib
import oracle

pytestmark = pytest.mark.gpu


def test_autotune_picks_valid_fast_options():
    beg, col = ib.gen_rmat(14, 16, seed=5)
    src = ib.sample_sources(beg, col, 256, seed=5)
    g = ib.Graph.from_csr(beg, col)
    try:
        best, gteps, log = g.autotune(src, reps=1)
        assert best.width in (32, 64, 128, 256)
        assert len(log) >= 10
        assert gteps >= log[0]["gteps"] * 0.999
        res = g.run(src, best)
        ref, _ = oracle.bfs(beg, col, src)
        assert np.array_equal(res.depth, ref)
    finally:
        g.close()
