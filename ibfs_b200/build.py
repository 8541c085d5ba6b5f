"""In-tree build of the native pieces.

``build_all()`` compiles
  * ``ibfs_b200/libibfs.so``  -- the C-ABI library (CUDA kernels for sm_100a
    + host C++), declared in ``include/ibfs.h``;
  * ``ibfs_b200/bin/gpu_ibfs`` -- the drop-in command line tool;
  * ``oracle/liboracle.so``   -- the CPU oracle (test infrastructure).

Everything is rebuilt only when a source is newer than its output.  nvcc
cross-compiles without a GPU, so this runs on CPU-only machines too.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp",
              "-Xptxas", "-O3", "--expt-relaxed-constexpr", f"-I{INCLUDE}"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", f"-I{INCLUDE}",
             "-I/usr/local/cuda/include"]

LIB_CU = ["engine.cu", "persistent_w32.cu", "persistent_w64.cu", "persistent_w128.cu",
          "persistent_w256.cu", "devloop.cu", "groupby_dev.cu", "convert.cu", "bytes_alg.cu",
          "server.cu", "serve_loop.cu", "noalloc.cu"]
LIB_CPP = ["host_graph.cpp", "autotune.cpp", "sink.cpp"]
HEADERS = ["bfs_device.cuh", "internal.h", "launch_common.cuh", "persistent.cuh"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build_lib(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(PKG, "libibfs.so")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ibfs.h")]
    objs = []
    jobs = []
    for f in LIB_CU:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdrs):
            jobs.append([_nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj])
    for f in LIB_CPP:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdrs):
            jobs.append(["g++", *CXX_FLAGS, "-c", src, "-o", obj])
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
    failed = None
    for cmd, pr in procs:
        o, _ = pr.communicate()
        if pr.returncode != 0 and failed is None:
            failed = (cmd, o)
    if failed:
        sys.stderr.write(failed[1])
        raise RuntimeError("build step failed: " + " ".join(failed[0]))
    if _newer(out, objs):
        _run([_nvcc(), *ARCH, "-shared", "-o", out, *objs, "-lgomp", "-lcudart"])
    return out


def build_cli(verbose: bool = False) -> str:
    src = os.path.join(CSRC, "cli.cpp")
    out_dir = os.path.join(PKG, "bin")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "gpu_ibfs")
    lib = os.path.join(PKG, "libibfs.so")
    if not os.path.exists(src):
        return out
    if _newer(out, [src, lib, os.path.join(INCLUDE, "ibfs.h")]):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", src, "-o", out, f"-L{PKG}", "-libfs",
              f"-Wl,-rpath,$ORIGIN/.."])
    # the edge-list converter's command line (tuple_text_to_bin)
    csrc = os.path.join(CSRC, "convert_cli.cpp")
    cout = os.path.join(out_dir, "tuple_text_to_bin")
    if os.path.exists(csrc) and _newer(cout, [csrc, lib, os.path.join(INCLUDE, "ibfs.h")]):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", csrc, "-o", cout, f"-L{PKG}", "-libfs",
              f"-Wl,-rpath,$ORIGIN/.."])
    return out


def build_oracle(verbose: bool = False) -> str:
    odir = os.path.join(ROOT, "oracle")
    src = os.path.join(odir, "oracle.c")
    out = os.path.join(odir, "liboracle.so")
    if _newer(out, [src]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-fopenmp", "-shared", src, "-o", out])
    return out


def build_ref(verbose: bool = False) -> str | None:
    """Compile the reference's host-side code into oracle/_ref (only where the
    reference sources are present; the GPU box uses the prebuilt binary)."""
    script = os.path.join(ROOT, "oracle", "build_ref.sh")
    if not os.path.exists(script):
        return None
    # where the reference sources are mounted in the build container
    ref = os.environ.get("IBFS_REFERENCE_DIR", "/root/reference")
    r = subprocess.run(["bash", script, ref], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if verbose:
        print(r.stdout)
    out = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    return out if os.path.exists(out) else None


def build_all(verbose: bool = False) -> None:
    build_lib(verbose)
    build_cli(verbose)
    build_oracle(verbose)
    build_ref(verbose)


if __name__ == "__main__":
    build_all(verbose=True)
