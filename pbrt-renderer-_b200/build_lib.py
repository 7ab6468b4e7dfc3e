"""Build recipe of the in-tree native libraries.

* ``csrc/libpt.so``  — the CUDA path tracer (sm_100a only) behind include/pt.h.
* ``host/libnori.so`` — the C++17 Nori plugin host (built by build_host()).

Run ``python pbrt-renderer-_b200/build_lib.py`` or ``__graft_entry__.build()``.
nvcc cross-compiles here without a GPU; the .so files travel with the tree.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd, quiet):
    if not quiet:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_libpt(quiet: bool = True, ptxas_verbose: bool = False) -> str:
    out = os.path.join(CSRC, "libpt.so")
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    for s in srcs:
        o = os.path.join(CSRC, "_obj", os.path.basename(s) + ".o")
        os.makedirs(os.path.dirname(o), exist_ok=True)
        cmd = [NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-c", s, "-o", o,
               "-I", os.path.join(ROOT, "include")]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        _run(cmd, quiet)
        objs.append(o)
    _run([NVCC, "-shared", *ARCH, "--cudart=static", "-o", out, *objs], quiet)
    return out


def build_host(quiet: bool = True) -> str | None:
    """C++17 Nori host library (XML scene loader + plugins) over libpt."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return None
    out = os.path.join(HOST, "libnori.so")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), "-I", HOST,
           "-I", CSRC, *srcs, "-o", out, "-L", CSRC, "-lpt", "-Wl,-rpath,$ORIGIN/../csrc"]
    _run(cmd, quiet)
    cli = os.path.join(HOST, "nori_render")
    main = os.path.join(HOST, "cli", "nori_render.cc")
    if os.path.exists(main):
        _run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", HOST, main, "-o", cli,
              "-L", HOST, "-lnori", "-L", CSRC, "-lpt", "-Wl,-rpath,$ORIGIN:$ORIGIN/../csrc"], quiet)
    return out


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build_libpt(quiet=False, ptxas_verbose=v))
    print(build_host(quiet=False))
