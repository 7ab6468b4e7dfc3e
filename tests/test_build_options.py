"""Build-time options of libpt that the default build does not compile.

PT_SHARED_STACK=k keeps the first k traversal-stack entries of each thread of
k_extend / k_shadow in shared memory (one column per thread) and the deeper
ones in local memory.  The default (0) keeps the whole stack in local memory,
which measured faster on B200; the option stays buildable so the choice can
be re-measured.  This cross-compiles the traversal kernels with the option
(nvcc needs no GPU) and checks the shared memory they then declare."""

import os
import re
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="nvcc not available")
@pytest.mark.parametrize("depth", [8])
def test_shared_stack_variant_compiles(depth):
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    src = os.path.join(ROOT, "pbrt-renderer-_b200", "csrc", "pt_render.cu")
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "pt_render_shared_stack.o")
        cmd = [nvcc, "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-c", src, "-o", out,
               "-I", os.path.join(ROOT, "include"), f"-DPT_SHARED_STACK={depth}", "-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        assert os.path.getsize(out) > 0
    # ptxas reports each kernel's properties after "Compiling entry function '<name>'"
    smem = {}
    name = None
    for line in r.stderr.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            name = m.group(1)
            continue
        m = re.search(r"Used \d+ registers.*?(\d+) bytes smem", line)
        if m and name:
            smem[name] = int(m.group(1))
    stack_bytes = depth * 256 * 8  # entries x threads per block x (base, mask)
    traversal = {k: v for k, v in smem.items() if "k_extend" in k or "k_shadow" in k}
    assert traversal, "no traversal kernels in the ptxas report"
    assert all(v >= stack_bytes for v in traversal.values()), traversal
