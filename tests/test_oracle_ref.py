"""The oracle pinned against the reference's own host code (CPU only).

tests/golden/*.npz were produced by tests/golden/make_golden.py, which ran
the reference's GroupBy, report, validate, deep_than_two and graph_reader
(compiled from the reference sources into oracle/_ref/ref_harness) and the
oracle, and checked the oracle depths against scipy.  These tests re-check
every recorded value; when the harness binary is present they also run it
live on freshly generated inputs.
"""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

import ibfs_b200 as ib
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def load(path):
    return dict(np.load(path))


def test_fixtures_present():
    names = {os.path.basename(f)[:-4] for f in FIXTURES}
    assert {"rmat_s10", "rmat_s12", "grid_32x32", "chunglu_3k", "edge_cases"} <= names


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_depths_match_golden(path):
    f = load(path)
    d, _ = oracle.bfs(f["beg"], f["col"], f["src"], 1)
    assert np.array_equal(d, f["depth"])


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_groupby_matches_reference(path):
    f = load(path)
    assert np.array_equal(oracle.groupby(f["beg"], f["col"], f["src"]), f["ref_groupby"])
    assert np.array_equal(ib.groupby_csr(f["beg"], f["col"], f["src"]), f["ref_groupby"])


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_teps_matches_reference_report(path):
    f = load(path)
    for i in range(len(f["src"])):
        row = f["depth"][i:i + 1]
        assert oracle.teps(f["beg"], row) == f["ref_report"][i][1]
        assert int((row != 255).sum()) == f["ref_report"][i][0]


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_reference_validate_accepts_oracle(path):
    f = load(path)
    assert np.all(f["ref_validate"] == 0)


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_deep_than_two_agrees(path):
    """deep_than_two (graph.cuh:28-70) is true iff no vertex sits at depth 2."""
    f = load(path)
    for i in range(len(f["src"])):
        assert bool(f["ref_deep2"][i]) == (not np.any(f["depth"][i] == 2))


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_loader_matches_reference(path, tmp_path):
    f = load(path)
    bp, cp = str(tmp_path / "b.bin"), str(tmp_path / "c.bin")
    ib.write_csr(bp, cp, f["beg"], f["col"])
    beg, col = ib.read_csr(bp, cp)
    assert np.array_equal(beg, f["ref_load_beg"].astype(np.int64))
    assert np.array_equal(col, f["ref_load_col"])


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_properties(path):
    """BFS properties the reference's validate intends (validate.h:13-19),
    checked correctly: d(src)=0, |d(u)-d(v)| <= 1 on reached edges, every
    reached non-source has a parent one level up, unreached stay INFTY."""
    f = load(path)
    beg, col, src, depth = f["beg"], f["col"], f["src"], f["depth"]
    V = len(beg) - 1
    rows = np.repeat(np.arange(V), np.diff(beg))
    for i, s in enumerate(src):
        d = depth[i].astype(np.int32)
        assert d[s] == 0
        du, dv = d[rows], d[col]
        both = (du != 255) & (dv != 255)
        assert np.all(np.abs(du[both] - dv[both]) <= 1)
        assert np.all((du != 255) == (dv != 255))  # reachability is closed under edges
        has_parent = np.zeros(V, bool)
        np.logical_or.at(has_parent, col[(du != 255)], (dv[(du != 255)] == du[(du != 255)] + 1))
        reached = (d != 255) & (np.arange(V) != s)
        assert np.all(has_parent[reached])


def test_bytes_alg_oracle_small():
    f = load(os.path.join(HERE, "golden", "edge_cases.npz"))
    b1 = oracle.bytes_alg(f["beg"], f["col"], f["depth"], 32)
    b2 = oracle.bytes_alg(f["beg"], f["col"], f["depth"], 64)
    V, n = len(f["beg"]) - 1, len(f["src"])
    assert b1 >= 2 * 4 * V + V * n and b2 > b1


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference harness not built here")
def test_live_reference_groupby_and_report():
    beg, col = ib.gen_rmat(11, 16, seed=77)
    src = ib.sample_sources(beg, col, 150, seed=9)
    with tempfile.TemporaryDirectory() as tmp:
        bp, cp = os.path.join(tmp, "b.bin"), os.path.join(tmp, "c.bin")
        ib.write_csr(bp, cp, beg, col)
        sp = os.path.join(tmp, "s.txt")
        np.savetxt(sp, src, fmt="%d")
        go = os.path.join(tmp, "g.txt")
        subprocess.run([HARNESS, "groupby", bp, cp, sp, go], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        assert np.array_equal(np.loadtxt(go, dtype=np.int32), oracle.groupby(beg, col, src))
        d, _ = oracle.bfs(beg, col, src, 1)
        dp = os.path.join(tmp, "d.u8")
        d.tofile(dp)
        out = subprocess.run([HARNESS, "report", bp, cp, dp, str(len(src))], check=True,
                             stdout=subprocess.PIPE, text=True).stdout
        rep = [ln.split() for ln in out.split("\n") if ln.strip() and ln.split()[0].isdigit()]
        for i, (nv, ne) in enumerate(rep):
            assert int(ne) == oracle.teps(beg, d[i:i + 1])
