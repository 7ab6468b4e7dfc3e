"""Build recipe for oracle/_ref/libref.so — the reference's own shader code on the CPU.

TEST INFRASTRUCTURE ONLY.  The reference renderer
(gracejinsotrue/PBRT-renderer-) runs its whole light transport in the HLSL
megakernel shaders/Shaders.hlsl and the .hlsli files it includes.  Those files
are plain shader arithmetic, so after a handful of mechanical rewrites they
compile as C++ against oracle/ref_shim/hlsl_cpu.h:

  * ``[shader("...")]`` and ``[loop]``/``[unroll]`` attributes are dropped;
  * ``: register(...)`` bindings are dropped and unsized resource arrays get a
    fixed size;
  * the ``cbuffer`` block's members become plain globals;
  * ``inout T x`` / ``out T x`` parameters become ``T& x`` (arrays stay arrays)
    and ``in`` is dropped;
  * the swizzles ``.xy``/``.xyz``/``.rgb`` become member calls;
  * ``float2(NextFloat(rng), NextFloat(rng))`` becomes brace-initialisation so
    the two draws happen left to right as in HLSL (C++ leaves the order of
    constructor arguments unspecified);
  * ``Texture2D`` (with or without a template argument) maps to the shim's
    ``Texture2D_t`` template.

The sources are read from the reference checkout (``--src``, default
/root/reference/shaders) and written to oracle/_ref/gen/; nothing from the
reference is copied into the repository.  ``MAX_BOUNCES`` is bound to a
run-time variable so one build serves every depth.  Literals are single
precision (``-fsingle-precision-constant``) and FP contraction is off, which
reproduces float32 HLSL arithmetic to the rounding of each libm call.
"""

from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")
SHIM = os.path.join(HERE, "ref_shim")
# the reference checkout: $PBRT_REFERENCE_ROOT, default /root/reference
REF_ROOT = os.environ.get("PBRT_REFERENCE_ROOT", "/root/reference")
DEFAULT_SRC = os.path.join(REF_ROOT, "shaders")

FILES = [
    "Common.hlsli", "RNG.hlsli", "GeometryUtils.hlsli", "RayQueryTrace.hlsli",
    "Microfacet.hlsli", "Disney.hlsli", "Hair.hlsli", "Material.hlsli",
    "Emitter.hlsli", "Envmap.hlsli", "Volume.hlsl", "Subsurface.hlsli",
    "Shaders.hlsl",
]


def rewrite(text: str) -> str:
    text = re.sub(r'\[shader\("[^"]*"\)\]', "", text)
    text = re.sub(r"\[(loop|unroll|branch|flatten)\]", "", text)
    text = re.sub(r":\s*register\([^)]*\)", "", text)
    text = re.sub(r"([\w<>]+)\s+(\w+)\[\]\s*;", r"\1 \2[64];", text)
    text = re.sub(r"cbuffer\s+\w+\s*\{(.*?)\};", r"\1", text, flags=re.S)
    ident = r"[A-Za-z_]\w*(?:<[^>]*>)?"
    text = re.sub(r"\b(?:inout|out)\s+(" + ident + r")\s+([A-Za-z_]\w*)\s*\[", r"\1 \2[", text)
    text = re.sub(r"\b(?:inout|out)\s+(" + ident + r")\s+([A-Za-z_]\w*)", r"\1& \2", text)
    text = re.sub(r"\bin\s+(" + ident + r")\s+([A-Za-z_]\w*)(\s*[,)])", r"\1 \2\3", text)
    text = re.sub(r"\.(xyz|rgb|xy)\b(?!\s*\()", r".\1()", text)
    text = text.replace("float2(NextFloat(rng), NextFloat(rng))", "float2{NextFloat(rng), NextFloat(rng)}")
    text = re.sub(r"\bTexture2D<", "Texture2D_t<", text)
    text = re.sub(r"\bTexture2D\b(?!_t)", "Texture2D_t<>", text)
    text = re.sub(r"\bTexture3D<", "Texture3D_t<", text)
    return text


def build(src: str = DEFAULT_SRC, quiet: bool = False) -> str:
    os.makedirs(GEN, exist_ok=True)
    for name in FILES:
        with open(os.path.join(src, name), encoding="utf-8") as f:
            text = f.read()
        with open(os.path.join(GEN, name), "w", encoding="utf-8") as f:
            f.write(rewrite(text))
    # libref.so: the reference's default build; libref_ris.so: its USE_RIS=1
    # build (resampled area-light NEE, shaders/Shaders.hlsl:481-488)
    lib = os.path.join(OUT, "libref.so")
    for name, extra in (("libref.so", []), ("libref_ris.so", ["-DUSE_RIS=1"])):
        cmd = [
            "g++", "-std=c++17", "-O2", "-march=x86-64-v2", "-mfma", "-ffp-contract=off",
            "-fsingle-precision-constant", "-fPIC", "-shared", "-w",
            "-DMAX_BOUNCES=g_max_bounces", *extra,
            "-I", GEN, "-I", SHIM,
            os.path.join(SHIM, "ref_entry.cpp"), "-o", os.path.join(OUT, name), "-lpthread",
        ]
        if not quiet:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    a = ap.parse_args()
    if not os.path.isdir(a.src):
        print(f"reference shaders not found at {a.src}", file=sys.stderr)
        sys.exit(1)
    print(build(a.src))
