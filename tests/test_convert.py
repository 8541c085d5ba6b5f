"""Edge-list text -> CSR conversion (the reference's tuple_text_to_bin).

CPU: a plain restatement of the reference converter's rules (token pairs,
ids shifted by the smallest id, lists in file order, both directions with
`reverse`) reproduces every golden case recorded from the reference binary
(tests/golden/make_convert_golden.py).  GPU: ibfs_convert_text writes the
same files byte for byte, and its clean mode equals a sorted, deduplicated,
symmetrised CSR without self loops.
"""
import os

import numpy as np
import pytest

import ibfs_b200 as ib

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "convert", "cases.npz")


def _cases():
    z = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in z.files})
    return [(n, z[n + "__text"].tobytes(), int(z[n + "__args"][0]), int(z[n + "__args"][1]),
             z[n + "__beg"], z[n + "__csr"]) for n in names]


def _tokens(text: bytes, skip: int):
    # header lines: the reference steps past offset 0 before looking for '\n'
    h, k = 0, 0
    while k < skip:
        h += 1
        if text[h:h + 1] == b"\n":
            h += 1
            k += 1
    return np.array([int(t) for t in text[h:].split()], np.int64)


def restate(text: bytes, reverse: int, skip: int):
    tok = _tokens(text, skip)
    vmin = tok.min()
    V = int(tok.max() - vmin + 1)
    u, v = tok[0::2] - vmin, tok[1::2] - vmin
    lists = [[] for _ in range(V)]
    for a, b in zip(u.tolist(), v.tolist()):
        lists[a].append(b)
        if reverse:
            # the reference writes both directions before counting either, so a
            # self loop lands twice in one slot and leaves the next one 0
            lists[b].append(a if a != b else 0)
    beg = np.zeros(V + 1, np.int64)
    beg[1:] = np.cumsum([len(x) for x in lists])
    col = np.array([x for lst in lists for x in lst], np.int64)
    return beg, col


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_restatement_matches_reference_fixture(case):
    name, text, rev, skip, beg, csr = case
    b, c = restate(text, rev, skip)
    assert np.array_equal(b, beg) and np.array_equal(c, csr)


def test_tiny_fixture_by_hand():
    z = np.load(GOLDEN)
    assert z["tiny_rev__beg"].tolist() == [0, 3, 6, 9, 11, 11, 12]
    assert z["tiny_rev__csr"].tolist() == [1, 2, 1, 0, 2, 0, 1, 0, 5, 3, 0, 2]


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_gpu_convert_matches_reference(case, tmp_path):
    name, text, rev, skip, beg, csr = case
    p = str(tmp_path / (name + ".txt"))
    with open(p, "wb") as f:
        f.write(text)
    bp, cp, V, E = ib.convert_text(p, reverse=bool(rev), skip_lines=skip)
    assert np.array_equal(np.fromfile(bp, "<u8").astype(np.int64), beg)
    assert np.array_equal(np.fromfile(cp, "<u8").astype(np.int64), csr)
    assert V == len(beg) - 1 and E == len(csr)


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_gpu_convert_clean(case, tmp_path):
    name, text, rev, skip, _, _ = case
    p = str(tmp_path / (name + ".txt"))
    with open(p, "wb") as f:
        f.write(text)
    bp, cp, V, E = ib.convert_text(p, reverse=bool(rev), skip_lines=skip, clean=True,
                                   out_prefix=str(tmp_path / "clean"))
    tok = _tokens(text, skip)
    vmin = tok.min()
    u, v = tok[0::2] - vmin, tok[1::2] - vmin
    pairs = np.unique(np.stack([np.concatenate([u, v]), np.concatenate([v, u])], 1), axis=0)
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    Vr = int(tok.max() - vmin + 1)
    beg = np.zeros(Vr + 1, np.int64)
    np.add.at(beg, pairs[:, 0] + 1, 1)
    beg = np.cumsum(beg)
    assert np.array_equal(np.fromfile(bp, "<u8").astype(np.int64), beg)
    assert np.array_equal(np.fromfile(cp, "<u8").astype(np.int64), pairs[:, 1])
    # and the files load as a graph whose traversals match the oracle
    b2, c2 = ib.read_csr(bp, cp)
    assert np.array_equal(b2, beg)


@pytest.mark.gpu
def test_gpu_convert_errors(tmp_path):
    p = str(tmp_path / "odd.txt")
    with open(p, "wb") as f:
        f.write(b"1 2\n3\n")
    with pytest.raises(ib.IbfsError) as ei:
        ib.convert_text(p)
    assert ei.value.status == 2
    with pytest.raises(ib.IbfsError) as ei:
        ib.convert_text(str(tmp_path / "missing.txt"))
    assert ei.value.status == 1


@pytest.mark.gpu
def test_gpu_convert_large_rmat(tmp_path):
    """A 1M-edge list through the multi-pass radix sort (4 digit passes)."""
    beg, col = ib.gen_rmat(17, 8, seed=9)
    V = len(beg) - 1
    src = np.repeat(np.arange(V), np.diff(beg))
    keep = src < col
    txt = "\n".join(f"{a} {b}" for a, b in zip(src[keep], col[keep])) + "\n"
    p = str(tmp_path / "g.txt")
    with open(p, "w") as f:
        f.write(txt)
    bp, cp, V2, E2 = ib.convert_text(p, reverse=True, clean=True)
    b2 = np.fromfile(bp, "<u8").astype(np.int64)
    c2 = np.fromfile(cp, "<u8").astype(np.int64)
    lo = int(min(src[keep].min(), col[keep].min()))
    # vertices below the smallest id in the file are shifted away
    assert V2 == int(max(src[keep].max(), col[keep].max())) - lo + 1
    assert np.array_equal(c2 + lo, col[beg[lo]:beg[lo + V2]])
