"""GPU path against the golden fixtures (reference-pinned, tests/golden/)."""
import glob
import os

import numpy as np
import pytest

import ibfs_b200 as ib

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("width", [32, 64, 128, 256])
def test_gpu_depths_match_golden(path, width):
    f = dict(np.load(path))
    g = ib.Graph.from_csr(f["beg"], f["col"])
    try:
        for mode in (ib.MODE_PLAIN, ib.MODE_PERSISTENT, ib.MODE_DEVICE_LOOP):
            res = g.run(f["src"], width=width, mode=mode, groupby=1)
            assert np.array_equal(res.depth, f["depth"])
            assert res.stats["traversed_edges"] == int(f["ref_report"][:, 1].sum())
        assert np.array_equal(g.groupby(f["src"]), f["ref_groupby"])
    finally:
        g.close()


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_from_reference_files(path, tmp_path):
    """The drop-in path: the reference's binary CSR files, loaded by the library."""
    f = dict(np.load(path))
    bp, cp = str(tmp_path / "x_beg_pos.bin"), str(tmp_path / "x_csr.bin")
    ib.write_csr(bp, cp, f["beg"], f["col"])
    g = ib.Graph.open(bp, cp)
    try:
        res = g.run(f["src"], width=128)
        assert np.array_equal(res.depth, f["depth"])
    finally:
        g.close()
