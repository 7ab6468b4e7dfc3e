"""The C++17 Nori host (host/libnori.so): XML scene loading through the
plugin registry, scene flattening and camera conversion, and a render through
the "path_mis" integrator, against the same scene built directly for libpt."""

import ctypes as C
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBNORI = os.path.join(ROOT, "pbrt-renderer-_b200", "host", "libnori.so")


def write_hdr(path, rgb):
    """Flat (non-RLE) Radiance RGBE file."""
    H, W = rgb.shape[:2]
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(f"-Y {H} +X {W}\n".encode())
        m = rgb.max(-1)
        e = np.where(m > 1e-32, np.ceil(np.log2(np.maximum(m, 1e-32))), -128).astype(np.int32)
        sc = np.where(m > 1e-32, 256.0 / np.exp2(e), 0.0)
        q = np.clip(np.floor(rgb * sc[..., None]), 0, 255).astype(np.uint8)
        ex = np.where(m > 1e-32, e + 128, 0).astype(np.uint8)
        f.write(np.concatenate([q, ex[..., None]], -1).tobytes())


def write_obj(path, v, f, with_normals=False):
    with open(path, "w") as o:
        for p in v:
            o.write(f"v {p[0]:.7g} {p[1]:.7g} {p[2]:.7g}\n")
        if with_normals:
            for p in v:
                o.write(f"vn {p[0]:.7g} {p[1]:.7g} {p[2]:.7g}\n")
        for t in f:
            if with_normals:
                o.write("f " + " ".join(f"{i + 1}//{i + 1}" for i in t) + "\n")
            else:
                o.write("f " + " ".join(str(i + 1) for i in t) + "\n")


SCENE_XML = """<?xml version="1.0"?>
<!-- generated test scene: a Disney sphere and a floor lit by a quad light -->
<scene>
  <string name="envmap" value="white.hdr"/>
  <float name="envmapScale" value="0.5"/>
  <integrator type="path_mis"><integer name="maxDepth" value="8"/></integrator>
  <camera type="perspective">
    <float name="fov" value="45"/>
    <transform name="toWorld"><lookat origin="0, 1.5, 5" target="0, 0.5, 0" up="0, 1, 0"/></transform>
    <integer name="width" value="64"/><integer name="height" value="48"/>
  </camera>
  <sampler type="independent"><integer name="sampleCount" value="4"/></sampler>
  <mesh type="obj">
    <string name="filename" value="sphere.obj"/>
    <transform name="toWorld"><scale value="0.8, 0.8, 0.8"/><translate value="0, 0.8, 0"/></transform>
    <bsdf type="disney">
      <color name="baseColor" value="0.8, 0.3, 0.2"/>
      <float name="roughness" value="0.4"/><float name="metallic" value="0.2"/><float name="clearcoat" value="0.5"/>
    </bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="floor.obj"/>
    <bsdf type="diffuse"><color name="albedo" value="0.6 0.6 0.6"/></bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="light.obj"/>
    <emitter type="area"><color name="radiance" value="8, 8, 8"/></emitter>
  </mesh>
</scene>
"""


@pytest.fixture(scope="module")
def scene_dir(tmp_path_factory, scenes):
    d = tmp_path_factory.mktemp("nori_scene")
    v, f = scenes.icosphere(3)
    write_obj(d / "sphere.obj", v, f, with_normals=True)
    write_obj(d / "floor.obj", np.array([[-3, 0, -3], [-3, 0, 3], [3, 0, 3], [3, 0, -3]], float),
              np.array([[0, 1, 2], [0, 2, 3]]))
    write_obj(d / "light.obj", np.array([[-0.5, 3, -0.5], [0.5, 3, -0.5], [0.5, 3, 0.5], [-0.5, 3, 0.5]], float),
              np.array([[0, 1, 2], [0, 2, 3]]))
    write_hdr(d / "white.hdr", np.ones((2, 4, 3), np.float32))
    (d / "scene.xml").write_text(SCENE_XML)
    return d


@pytest.fixture(scope="module")
def nori():
    L = C.CDLL(LIBNORI)
    L.nori_load.restype = C.c_void_p
    L.nori_load.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
    L.nori_free.argtypes = [C.c_void_p]
    L.nori_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.nori_camera.argtypes = [C.c_void_p, C.c_void_p]
    L.nori_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    L.nori_materials.restype = C.c_uint32
    L.nori_render.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                              C.c_size_t]
    L.nori_flat.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.nori_flat.restype = C.c_uint64
    return L


def load(nori, path):
    err = C.create_string_buffer(512)
    h = nori.nori_load(str(path).encode(), err, 512)
    return h, err.value.decode()


def test_load_and_flatten(nori, pt, scene_dir):
    h, err = load(nori, scene_dir / "scene.xml")
    assert h, err
    info = (C.c_uint32 * 8)()
    nori.nori_info(h, info)
    assert list(info) == [64, 48, 4, 3, 1280 + 2 + 2, 1, 0, 8]
    mats = (pt.pt_material * 3)()
    assert nori.nori_materials(h, mats, 3) == 3
    assert mats[0].type == pt.PT_MAT_DISNEY and abs(mats[0].clearcoat - 0.5) < 1e-7
    assert abs(mats[0].specular - 0.5) < 1e-7 and abs(mats[0].sheenTint - 0.5) < 1e-7  # Disney defaults
    assert mats[1].type == pt.PT_MAT_DIFFUSE and abs(mats[1].albedo[0] - 0.6) < 1e-7
    assert mats[2].isEmitter == 1 and list(mats[2].radiance) == [8.0, 8.0, 8.0]
    assert mats[1].indexOffset == mats[0].indexCount and mats[2].vertexOffset == mats[0].vertexCount + 4
    cam = pt.pt_camera()
    nori.nori_camera(h, C.byref(cam))
    pos = np.array(cam.pos)
    assert np.allclose(pos, [0, 1.5, 5], atol=1e-5)
    ctr = np.array(cam.llc) + 0.5 * np.array(cam.horizontal) + 0.5 * np.array(cam.vertical) - pos
    fwd = np.array([0, -1.0, -5.0]) / math.sqrt(26)
    assert np.allclose(ctr / np.linalg.norm(ctr), fwd, atol=1e-4)
    # Nori's fov is along X: |horizontal| = 2 tan(22.5 deg) at unit distance, |vertical| = that / aspect
    assert abs(np.linalg.norm(cam.horizontal) - 2 * math.tan(math.radians(22.5))) < 1e-4
    assert abs(np.linalg.norm(cam.vertical) - 2 * math.tan(math.radians(22.5)) * 48 / 64) < 1e-4
    # flattened buffers: the sphere's OBJ normals went through the transform's
    # inverse transpose (a uniform scale) and were renormalised
    pos, nrm, idx, env = flat(nori, h, 0), flat(nori, h, 1), flat(nori, h, 4), flat(nori, h, 5)
    assert len(idx) == 3 * 1284 and idx.max() < len(pos) // 3
    nv = mats[0].vertexCount
    p = pos.reshape(-1, 3)[:nv]
    assert np.allclose(nrm.reshape(-1, 3)[:nv], (p - [0, 0.8, 0]) / 0.8, atol=1e-5)
    assert np.allclose(pos.reshape(-1, 3)[nv:nv + 4], [[-3, 0, -3], [-3, 0, 3], [3, 0, 3], [3, 0, -3]])
    assert nori.nori_flat(h, 6, None) == 4 and env.size == 2 * 4 * 3 and np.allclose(env, 1.0, rtol=1e-2)
    nori.nori_free(h)


@pytest.mark.parametrize("bad,msg", [
    ("<scene><bogus/></scene>", "unexpected tag"),
    ("<scene><camera type='perspective'><float name='fov' value='abc'/></camera></scene>", "floating point"),
    ("<scene><mesh type='obj'><string name='filename' value='missing.obj'/></mesh></scene>", "Unable to open OBJ"),
    ("<scene><integrator type='nonexistent'/></scene>", "could not be found"),
    ("<scene></scene>", "No camera"),
    ("<scene><float name='x' value='1' extra='2'/></scene>", "unexpected attribute"),
])
def test_parse_errors_are_reported(nori, tmp_path, bad, msg):
    p = tmp_path / "bad.xml"
    p.write_text(bad)
    h, err = load(nori, p)
    assert not h and msg in err, err


@pytest.mark.gpu
def test_xml_render_matches_direct_scene(nori, pt, scenes, scene_dir):
    """The XML path (parser -> plugins -> flatten -> camera) renders the same
    image as the scene assembled by hand for libpt."""
    h, err = load(nori, scene_dir / "scene.xml")
    assert h, err
    W, H = 64, 48
    s = np.zeros((H, W, 4), np.float32)
    c = np.zeros_like(s)
    st = pt.pt_stats()
    e = C.create_string_buffer(512)
    assert nori.nori_render(h, 4, 0, s.ctypes.data, c.ctypes.data, C.byref(st), e, 512) == 0, e.value
    assert st.paths == W * H * 4 and np.all(s[..., 3] == 4)
    # the same flattened arrays, material records and camera through libpt directly
    mats = (pt.pt_material * 3)()
    nori.nori_materials(h, mats, 3)
    cam = pt.pt_camera()
    nori.nori_camera(h, C.byref(cam))
    arrays = [flat(nori, h, k) for k in range(6)]
    pos, nrm, uv, tan, idx, env = arrays
    ew = int(nori.nori_flat(h, 6, None))
    # geometry as written in the OBJ files, placed by the toWorld transform (the
    # OBJ loader renumbers vertices by first use, so compare triangle corners)
    v, f = scenes.icosphere(3)
    assert len(pos) == 3 * (len(v) + 8) and len(idx) == 3 * (len(f) + 4)
    corners = pos.reshape(-1, 3)[idx[:f.size]]
    assert np.allclose(corners, (np.asarray(v) * 0.8 + [0, 0.8, 0])[f.reshape(-1)], atol=1e-6)
    sc = pt.Scene(pos, idx, list(mats), normals=nrm if nrm.size else None, texcoords=uv if uv.size else None,
                  tangents=tan if tan.size else None, env_rgb=env.reshape(-1, ew, 3), env_scale=0.5)
    ctx = pt.Context(0)
    ctx.upload(sc)
    d, _, _ = ctx.render(pt.render_params(W, H, 4, cam, max_depth=8))
    ctx.close()
    assert np.array_equal(s, d), np.abs(s - d).max()
    nori.nori_free(h)


def flat(nori, h, which):
    n = int(nori.nori_flat(h, which, None))
    a = np.zeros(n, np.uint32 if which == 4 else np.float32)
    nori.nori_flat(h, which, a.ctypes.data)
    return a
