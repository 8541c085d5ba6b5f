"""Generate tests/golden/convert/cases.npz from the reference's own edge-list
converter (tuple_text_to_bin.cpp, built by oracle/build_ref.sh into
oracle/_ref/tuple_text_to_bin):

    python tests/golden/make_convert_golden.py

For every case it stores the input text, the converter's arguments and the
reference's _beg_pos.bin / _csr.bin contents.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
CONV = os.path.join(ROOT, "oracle", "_ref", "tuple_text_to_bin")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "convert", "cases.npz")


def cases():
    yield "tiny_rev", b"0 1\n1 2\n2 0\n3 3\n1 0\n5 2\n", 1, 0
    yield "tiny_fwd", b"0 1\n1 2\n2 0\n3 3\n1 0\n5 2\n", 0, 0
    rng = np.random.default_rng(7)
    m = 2000
    u = rng.integers(5, 400, m)
    v = rng.integers(5, 400, m)
    v[::37] = u[::37]                     # self loops
    u[100:140], v[100:140] = u[:40], v[:40]  # duplicates
    seps = [b" ", b"\t", b"  ", b" \t"]
    lines = [b"# header one", b"% header two"]
    for i in range(m):
        lines.append(str(u[i]).encode() + seps[i % 4] + str(v[i]).encode())
    yield "rand_rev_skip2", b"\n".join(lines) + b"\n", 1, 2
    m = 60000
    u = rng.integers(0, 30000, m)
    v = rng.integers(0, 30000, m)
    txt = b"".join(b"%d %d\n" % (a, b) for a, b in zip(u, v))
    yield "rand_fwd_60k", txt, 0, 0


def main():
    if not os.path.exists(CONV):
        raise SystemExit("oracle/_ref/tuple_text_to_bin missing: run oracle/build_ref.sh")
    rec = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, text, rev, skip in cases():
            p = os.path.join(tmp, name + ".txt")
            with open(p, "wb") as f:
                f.write(text)
            subprocess.run([CONV, p, str(rev), str(skip)], check=True, cwd=tmp,
                           stdout=subprocess.DEVNULL)
            rec[name + "__text"] = np.frombuffer(text, np.uint8)
            rec[name + "__args"] = np.array([rev, skip], np.int64)
            rec[name + "__beg"] = np.fromfile(p + "_beg_pos.bin", "<u8").astype(np.int64)
            rec[name + "__csr"] = np.fromfile(p + "_csr.bin", "<u8").astype(np.int64)
            print(name, "V", len(rec[name + "__beg"]) - 1, "E", len(rec[name + "__csr"]))
    np.savez_compressed(OUT, **rec)


if __name__ == "__main__":
    main()
