"""CPU checks of the C ABI library: it loads, exports every entry point that
include/ibfs.h declares, and its host-only paths (generators, file formats,
source files, argument and error handling) behave -- no kernel launches."""
import os
import re

import numpy as np
import pytest

import ibfs_b200 as ib
from ibfs_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "ibfs.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ibfs_[a-z_0-9]+)\s*\(", txt)))


def test_header_symbols_exported():
    lib = api._lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ibfs.h but not exported"
    # and the Python binding covers every one of them
    assert set(names) <= set(api.exported_names())


def test_strerror_and_version():
    lib = api._lib()
    for s in range(0, 11):
        assert lib.ibfs_strerror(s)
    assert b"sm_100a" in lib.ibfs_version()


def test_opts_default_matches_reference_constants():
    o = ib.default_opts()
    assert o.width == 128  # comp_t = uint4 (comm.h:44)
    assert o.sml_shed == 32 and o.lrg_shed == 512  # ibfs.cu:71-72
    assert o.switch_level == -1
    assert o.alpha == 4.0 and o.beta == 24.0


def test_rmat_deterministic_and_clean():
    b1, c1 = ib.gen_rmat(10, 16, seed=3)
    b2, c2 = ib.gen_rmat(10, 16, seed=3)
    b3, _ = ib.gen_rmat(10, 16, seed=4)
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    assert not np.array_equal(b1, b3)
    V = len(b1) - 1
    for v in range(V):
        a = c1[b1[v]:b1[v + 1]]
        assert np.all(np.diff(a) > 0)  # sorted, no duplicates
        assert not np.any(a == v)  # no self loops
    # symmetric
    src = np.repeat(np.arange(V), np.diff(b1))
    fwd = set(zip(src.tolist(), c1.tolist()))
    assert all((y, x) in fwd for x, y in fwd)


def test_grid_generator_counts():
    beg, col = ib.gen_grid(32, 32, 0.0, 0.0, seed=1)
    assert len(beg) - 1 == 1024
    assert len(col) == 2 * (2 * 32 * 31)
    beg, col = ib.gen_grid(64, 64, 0.05, 0.001, seed=4)
    und = len(col) // 2
    base = 2 * 64 * 63
    assert 0.9 * base < und < base


def test_chung_lu_degrees():
    beg, col = ib.gen_chung_lu(20000, 400000, 2.1, 2000.0, seed=5)
    deg = np.diff(beg)
    assert deg.max() <= 2100 and deg.max() > 500
    assert 25 < deg.mean() < 45


def test_csr_files_roundtrip(tmp_path):
    beg, col = ib.gen_rmat(8, 8, seed=2)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    ib.write_csr(bp, cp, beg, col)
    raw_b = np.fromfile(bp, dtype="<u8")
    raw_c = np.fromfile(cp, dtype="<u8")
    assert np.array_equal(raw_b, beg.astype(np.uint64))
    assert np.array_equal(raw_c, col.astype(np.uint64))
    assert raw_b[-1] == len(raw_c)  # begin[V] = E (tuple_text_to_bin.cpp:149-152)


def _open_status(bp, cp):
    import ctypes as C

    h = C.c_void_p()
    return api._lib().ibfs_graph_open(bp.encode(), cp.encode(), 0, C.byref(h))


def test_loader_errors(tmp_path):
    beg, col = ib.gen_rmat(6, 4, seed=2)
    bp, cp = str(tmp_path / "b.bin"), str(tmp_path / "c.bin")
    ib.write_csr(bp, cp, beg, col)
    assert _open_status(str(tmp_path / "missing.bin"), cp) == 1  # IO
    # truncated csr: beg[V] != E
    np.fromfile(cp, dtype="<u8")[:-3].tofile(str(tmp_path / "short.bin"))
    assert _open_status(bp, str(tmp_path / "short.bin")) == 2  # FORMAT
    # size not a multiple of 8
    with open(str(tmp_path / "odd.bin"), "wb") as f:
        f.write(b"\x00" * 13)
    assert _open_status(bp, str(tmp_path / "odd.bin")) == 2
    # a column id >= V
    bad = np.fromfile(cp, dtype="<u8")
    bad[0] = len(beg) + 5
    bad.tofile(str(tmp_path / "bad.bin"))
    assert _open_status(bp, str(tmp_path / "bad.bin")) == 2
    # non-monotone offsets
    bb = np.fromfile(bp, dtype="<u8")
    bb[1], bb[2] = bb[2] + 1, bb[1]
    bb.tofile(str(tmp_path / "nm.bin"))
    assert _open_status(str(tmp_path / "nm.bin"), cp) == 2


def test_source_file_roundtrip(tmp_path):
    p = str(tmp_path / "src.dat")
    ids = np.array([5, 0, 17, 17, 3], np.int32)
    ib.write_src_v(p, ids)
    assert np.array_equal(ib.read_src_v(p), ids)
    with open(p, "a") as f:
        f.write("\n  \n42\n")
    assert ib.read_src_v(p).tolist() == [5, 0, 17, 17, 3, 42]
    with open(p, "a") as f:
        f.write("x1\n")
    with pytest.raises(ib.IbfsError) as ei:
        ib.read_src_v(p)
    assert ei.value.status == 2


def test_sample_sources():
    beg, col = ib.gen_rmat(10, 16, seed=1)
    s = ib.sample_sources(beg, col, 200, seed=1)
    assert len(set(s.tolist())) == 200
    assert np.all(np.diff(beg)[s] > 0)
    s2 = ib.sample_sources(beg, col, 200, seed=1, giant_component=True)
    assert len(set(s2.tolist())) == 200
    with pytest.raises(ib.IbfsError):
        ib.sample_sources(beg, col, 10**6, seed=1)


def test_csr_from_edges_rejects_bad_ids():
    with pytest.raises(ib.IbfsError) as ei:
        ib.csr_from_edges(np.array([0, 5]), np.array([1, 2]), 3)
    assert ei.value.status == 3



def test_groupby_maxhub_variant_rule():
    """The largest-hub GroupBy variant (groupby = 3) against a plain Python
    statement of its rule: eligible sources (degree <= 128 with a neighbour
    above 128) first, keyed by their highest-degree such neighbour (ties:
    smaller id), largest hubs first and stable; the rest after, in input
    order."""
    beg, col = ib.gen_rmat(11, 16, seed=17)
    deg = np.diff(beg)
    rng = np.random.default_rng(3)
    src = rng.integers(0, len(deg), 500).astype(np.int32)

    def hub(s):
        if deg[s] > 128:
            return -1
        best, h = 128, -1
        for u in col[beg[s]:beg[s + 1]].tolist():
            if deg[u] > best or (deg[u] == best and best > 128 and u < h):
                best, h = deg[u], u
        return h

    hubs = [hub(s) for s in src.tolist()]
    elig = sorted((i for i in range(len(src)) if hubs[i] >= 0),
                  key=lambda i: (-deg[hubs[i]], hubs[i]))
    ref = np.array([src[i] for i in elig] + [src[i] for i in range(len(src)) if hubs[i] < 0],
                   np.int32)
    assert len(elig) > 50
    assert np.array_equal(ib.groupby_csr_maxhub(beg, col, src), ref)


def test_server_arena_rows_clamped_to_int32():
    """Output rows reach the kernels as int32 indices: the arena's row count
    is capped at INT32_MAX however small the rows are."""
    from ibfs_b200 import api

    rows = api._lib().ibfs_server_arena_rows
    assert rows(1000, 10, 1) == 100
    assert rows(1000, 10, 2) == 50
    assert rows(1 << 40, 1, 1) == 2**31 - 1
    assert rows(1 << 34, 8, 2) == (1 << 34) // 16
    assert rows(0, 10, 1) == 0 and rows(100, 0, 1) == 0 and rows(100, 10, 3) == 0
