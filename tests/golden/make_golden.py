"""Generate the golden fixtures in tests/golden/*.npz.

Run from the repository root after ``python __graft_entry__.py`` has built
oracle/_ref/ref_harness from the reference sources:

    python tests/golden/make_golden.py

For every case it writes the graph in the reference's binary CSR format and
records what the REFERENCE's own host code computes on it (through
oracle/_ref/ref_harness):
  * ref_load_beg / ref_load_col -- graph_reader's narrowed arrays
                                   (graph_reader.cuh:63-119);
  * ref_groupby                 -- GroupBy's source order (GroupBy.cuh:6-115);
  * ref_report                  -- report's (vertices, edges) per source row
                                   (validate.h:59-76) on the oracle depths;
  * ref_validate                -- validate's return code per row
                                   (validate.h:2-56);
  * ref_deep2                   -- deep_than_two per source (graph.cuh:28-70).
and the oracle's per-source depths (oracle/oracle.c), which this script also
checks against scipy's breadth-first shortest paths before saving.
The reference has no complete CPU BFS, so the depth arrays are pinned by the
oracle + scipy agreement, and GroupBy / report / validate / deep_than_two /
the loader are pinned by the reference itself.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import ibfs_b200 as ib  # noqa: E402
import oracle  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
OUT_DIR = os.path.dirname(os.path.abspath(__file__))


def edge_case_graph():
    e = [(0, 1), (1, 2), (2, 3), (3, 0), (0, 0), (0, 1), (4, 5), (5, 6)]
    e += [(7, i) for i in range(8, 140)]          # a hub of degree > 128
    e += [(8, 9), (9, 10), (10, 11)]
    e += [(150 + i, 7) for i in range(5)]          # low-degree sources next to the hub
    u = np.array([a for a, _ in e], np.int32)
    v = np.array([b for _, b in e], np.int32)
    beg, col = ib.csr_from_edges(u, v, 160)       # 140..149, 155..159 isolated
    src = np.array([0, 145, 4, 7, 7, 150, 151, 11, 2, 0, 152, 153, 154, 9], np.int32)
    return beg, col, src


def cases():
    beg, col = ib.gen_rmat(10, 16, seed=11)
    yield "rmat_s10", beg, col, ib.sample_sources(beg, col, 200, seed=3)
    beg, col = ib.gen_rmat(12, 16, seed=1)
    yield "rmat_s12", beg, col, ib.sample_sources(beg, col, 128, seed=1)
    beg, col = ib.gen_grid(32, 32, 0.05, 0.001, seed=4)
    yield "grid_32x32", beg, col, ib.sample_sources(beg, col, 64, seed=4)
    beg, col = ib.gen_chung_lu(3000, 60000, 2.1, 600.0, seed=5)
    yield "chunglu_3k", beg, col, ib.sample_sources(beg, col, 96, seed=5)
    beg, col, src = edge_case_graph()
    yield "edge_cases", beg, col, src


def harness(*args, cwd=None) -> str:
    """Run the harness; drop the reference's own log lines (non-numeric)."""
    r = subprocess.run([HARNESS, *args], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                       text=True, cwd=cwd, check=True)
    keep = [ln for ln in r.stdout.split("\n")
            if ln.strip() and all(t.lstrip("-").isdigit() for t in ln.split())]
    return "\n".join(keep)


def scipy_depths(beg, col, src):
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg

    V = len(beg) - 1
    A = sp.csr_matrix((np.ones(len(col), np.int8), col, beg), shape=(V, V))
    d = cg.shortest_path(A, unweighted=True, indices=src)
    return np.where(np.isinf(d), 255, d).astype(np.uint8)


def record(name, beg, col, src, tmp):
    bp, cp = os.path.join(tmp, f"{name}_beg_pos.bin"), os.path.join(tmp, f"{name}_csr.bin")
    ib.write_csr(bp, cp, beg, col)
    V = len(beg) - 1
    # loader
    ob, oc = os.path.join(tmp, "ld_beg.i32"), os.path.join(tmp, "ld_csr.i32")
    harness("load", bp, cp, ob, oc)
    ref_beg = np.fromfile(ob, np.int32)
    ref_col = np.fromfile(oc, np.int32)
    # groupby (writes origin_source.dat / new_source.dat into its cwd)
    sp_ = os.path.join(tmp, "src.txt")
    np.savetxt(sp_, src, fmt="%d")
    gout = os.path.join(tmp, "grouped.txt")
    harness("groupby", bp, cp, sp_, gout, cwd=tmp)
    ref_groupby = np.loadtxt(gout, dtype=np.int32, ndmin=1)
    # oracle depths, checked against scipy
    depth, _ = oracle.bfs(beg, col, src, 1)
    assert np.array_equal(depth, scipy_depths(beg, col, src)), name
    dp = os.path.join(tmp, "depth.u8")
    depth.tofile(dp)
    rep = np.array([[int(x) for x in ln.split()] for ln in harness("report", bp, cp, dp,
                                                                    str(len(src))).split("\n")
                    if ln.strip()], np.int64)
    val = np.array([int(x) for x in harness("validate", bp, cp, dp, str(len(src))).split()],
                   np.int32)
    deep2 = np.array([int(x) for x in harness("deep2", bp, cp, sp_).split()], np.int32)
    np.savez_compressed(os.path.join(OUT_DIR, f"{name}.npz"), beg=beg, col=col, src=src,
                        depth=depth, ref_load_beg=ref_beg, ref_load_col=ref_col,
                        ref_groupby=ref_groupby, ref_report=rep, ref_validate=val,
                        ref_deep2=deep2)
    print(f"{name}: V={V} E={len(col)} n={len(src)} maxlevel="
          f"{int(depth[depth != 255].max())} validate={sorted(set(val.tolist()))}")


def main():
    if not os.path.exists(HARNESS):
        sys.exit("oracle/_ref/ref_harness missing: build it with oracle/build_ref.sh")
    with tempfile.TemporaryDirectory() as tmp:
        for name, beg, col, src in cases():
            record(name, beg, col, np.asarray(src, np.int32), tmp)


if __name__ == "__main__":
    main()
