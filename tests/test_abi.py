"""The C ABI boundary (include/pt.h) without a GPU: the library loads, exports
every entry point the header declares, the ctypes mirrors have the C layout,
and calls fail with status codes (never a crash) where no device exists."""

import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pt.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(pt_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["pt_create", "pt_destroy", "pt_last_error", "pt_upload_scene", "pt_render", "pt_bsdf_eval_batch",
              "pt_bsdf_sample_batch", "pt_trace_closest", "pt_trace_shadow", "pt_bvh_read"]:
        assert n in names


def test_library_exports_every_declared_symbol(pt):
    lib = C.CDLL(pt.LIBPT_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_c(pt):
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "pt.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(pt_material), sizeof(pt_volume),
         sizeof(pt_grid), sizeof(pt_scene_desc), sizeof(pt_camera), sizeof(pt_render_params), sizeof(pt_film),
         sizeof(pt_stats), sizeof(pt_hit), sizeof(pt_texture), sizeof(pt_cache_params), sizeof(pt_cache_stats),
         sizeof(pt_request), sizeof(pt_batch_tuning));
  printf("%zu %zu %zu %zu %zu\n", offsetof(pt_material, roughness), offsetof(pt_scene_desc, env_rgb),
         offsetof(pt_render_params, camera), offsetof(pt_scene_desc, textures), offsetof(pt_texture, srgb));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in out[0].split()]
    offs = [int(x) for x in out[1].split()]
    py = [C.sizeof(t) for t in (pt.pt_material, pt.pt_volume, pt.pt_grid, pt.pt_scene_desc, pt.pt_camera,
                                pt.pt_render_params, pt.pt_film, pt.pt_stats, pt.pt_hit, pt.pt_texture,
                                pt.pt_cache_params, pt.pt_cache_stats, pt.pt_request, pt.pt_batch_tuning)]
    assert sizes == py
    assert offs == [pt.pt_material.roughness.offset, pt.pt_scene_desc.env_rgb.offset,
                    pt.pt_render_params.camera.offset, pt.pt_scene_desc.textures.offset, pt.pt_texture.srgb.offset]


def test_null_and_invalid_arguments_fail_cleanly(pt):
    lib = pt.lib()
    assert lib.pt_create(None, 0) == -1                   # PT_E_INVALID
    assert lib.pt_destroy(None) == -1
    assert lib.pt_upload_scene(None, None) == -1
    assert lib.pt_render(None, None, None, None) == -1
    assert lib.pt_last_error(None) == b"null context"


def test_create_without_device_reports_cuda_error(pt):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = pt.lib().pt_create(C.byref(h), 0)
    assert rc == -2 and not h.value   # PT_E_CUDA, no context handed out
