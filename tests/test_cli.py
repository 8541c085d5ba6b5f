"""The gpu_ibfs command line (drop-in for the reference's gpu-ibfs)."""
import os
import subprocess

import numpy as np
import pytest

import ibfs_b200 as ib

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLI = os.path.join(ROOT, "ibfs_b200", "bin", "gpu_ibfs")


@pytest.fixture(scope="module", autouse=True)
def _cli():
    from ibfs_b200 import build

    build.build_lib()
    build.build_cli()


def test_wrong_input_exits_like_reference():
    r = subprocess.run([CLI, "a", "b"], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 255  # exit(-1), ibfs.cu:63
    assert "Wrong input" in r.stdout
    r = subprocess.run([CLI, "a", "b", "128", "2", "128", "--bogus"], stdout=subprocess.PIPE,
                       text=True)
    assert r.returncode == 255


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["--groupby", "--batched"], ["--plain"],
                                   ["--width", "64", "--alpha", "4"],
                                   ["--device-loop", "--td-stage", "--bu-filter", "1"],
                                   ["--device-loop", "--sparse-push", "4"]])
def test_cli_depths_match_golden(tmp_path, extra):
    f = dict(np.load(os.path.join(HERE, "golden", "rmat_s10.npz")))
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    ib.write_csr(bp, cp, f["beg"], f["col"])
    sp = str(tmp_path / "src.dat")
    ib.write_src_v(sp, f["src"])
    out = str(tmp_path / "depth.bin")
    conc = "64" if "64" in extra else "128"
    r = subprocess.run([CLI, bp, cp, conc, "-1", str(len(f["src"])), "--sources", sp,
                        "--depth-out", out, *extra], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 0, r.stdout
    assert "Traversal-" in r.stdout
    got = np.fromfile(out, np.uint8).reshape(len(f["src"]), -1)
    assert np.array_equal(got, f["depth"])


@pytest.mark.gpu
def test_cli_generated_sources_and_fixed_switch(tmp_path):
    beg, col = ib.gen_rmat(9, 8, seed=3)
    bp, cp = str(tmp_path / "b.bin"), str(tmp_path / "c.bin")
    ib.write_csr(bp, cp, beg, col)
    r = subprocess.run([CLI, bp, cp, "128", "2", "256"], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 0, r.stdout
    assert r.stdout.count("Traversal-iter-") == 2
