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
        # shared exponent e from frexp (max = f * 2^e, f in [0.5, 1)): mantissas
        # rgb * 256 / 2^e < 256, so 1.0 is stored exactly as 128 at e = 1
        m = rgb.max(-1)
        _, e = np.frexp(np.maximum(m, 1e-32))
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


def nori_lib():
    """ctypes binding of the Nori host's C surface (host/capi.cpp)."""
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
    L.nori_env_scale.argtypes = [C.c_void_p]
    L.nori_env_scale.restype = C.c_float
    return L


@pytest.fixture(scope="module")
def nori():
    return nori_lib()


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
    # nesting rules of the format
    ("<float name='x' value='1'/>", "cannot be the document element"),
    ("<scene><mesh type='obj'><transform name='toWorld'><float name='x' value='1'/></transform></mesh></scene>",
     "holds transform steps only"),
    ("<scene><mesh type='obj'><scale value='2'/></mesh></scene>", "must appear inside <transform>"),
    ("<scene><float name='x' value='1'><float name='y' value='2'/></float></scene>",
     "must appear inside a scene object"),
    ("<scene><mesh type='obj'><transform name='toWorld'><mesh type='obj'/></transform></mesh></scene>",
     "holds transform steps only"),
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


def write_hair(path, strands, thickness=None, default_thickness=0.1, default_segments=None):
    """A HAIR file (Cem Yuksel's format): 128-byte header, then the segment
    counts (u16 per strand, omitted when all strands have default_segments),
    points (3 x f32), optional thickness (f32 per point)."""
    import struct

    flags = 2 | (0 if default_segments is not None else 1) | (4 if thickness is not None else 0)
    npts = sum(len(s) for s in strands)
    hdr = struct.pack("<4sIIIIff3f", b"HAIR", len(strands), npts, flags, default_segments or 0,
                      default_thickness, 1.0, 1.0, 1.0, 1.0)
    hdr += b"\0" * (128 - len(hdr))
    with open(path, "wb") as f:
        f.write(hdr)
        if default_segments is None:
            f.write(np.array([len(s) - 1 for s in strands], np.uint16).tobytes())
        f.write(np.concatenate([np.asarray(s, np.float32).reshape(-1) for s in strands]).tobytes())
        if thickness is not None:
            f.write(np.asarray(thickness, np.float32).tobytes())


def wavy_strands(n=40, segs=10, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        x0, y0 = rng.uniform(-2, 2), rng.uniform(-0.5, 0.5)
        z = np.linspace(-4, 4, segs + 1)
        out.append(np.stack([x0 + 0.3 * np.sin(z * 1.5 + k), y0 + 0 * z, z], 1))
    return out


HAIR_XML = """<scene>
  <integrator type="path_mis"/>
  <camera type="perspective">
    <float name="fov" value="55"/>
    <transform name="toWorld"><lookat target="0, 0, 0" origin="0, 12, 0" up="0, 0, 1"/></transform>
    <integer name="height" value="48"/><integer name="width" value="64"/>
  </camera>
  <sampler type="independent"><integer name="sampleCount" value="64"/></sampler>
  <mesh type="hair">
    <string name="filename" value="strands.hair"/>
    <integer name="sides" value="{sides}"/>
    <float name="radiusScale" value="{scale}"/>
    <bsdf type="hair_bsdf">
      <color name="color" value="1.0 1.0 1.0"/>
      <float name="beta_m" value="0.2"/><float name="beta_n" value="0.3"/>
      <float name="alpha" value="2.0"/><float name="eta" value="1.55"/>
    </bsdf>
  </mesh>
</scene>
"""


@pytest.fixture(scope="module")
def hair_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("hair_scene")
    strands = wavy_strands()
    thick = np.concatenate([np.linspace(0.12, 0.04, len(s)) for s in strands])
    write_hair(d / "strands.hair", strands, thickness=thick)
    (d / "textures").mkdir()
    write_hdr(d / "textures" / "white_furnace.hdr", np.ones((2, 2, 3), np.float32))  # the scene's default envmap
    (d / "scene.xml").write_text(HAIR_XML.format(sides=6, scale=1.0))
    return d, strands, thick


def test_hair_tessellation(nori, pt, hair_dir):
    d, strands, thick = hair_dir
    h, err = load(nori, d / "scene.xml")
    assert h, err
    S = 6
    nv = sum(len(s) for s in strands) * S
    nt = sum(len(s) - 1 for s in strands) * 2 * S
    info = (C.c_uint32 * 8)()
    nori.nori_info(h, info)
    assert info[4] == nt and info[7] == 32  # path_mis default depth
    pos, nrm, uv, tan = (flat(nori, h, k).reshape(-1, w) for k, w in ((0, 3), (1, 3), (2, 2), (3, 3)))
    assert len(pos) == nv and len(tan) == nv
    centres = np.concatenate(strands).repeat(S, 0)
    radii = np.repeat(thick * 0.5, S)
    # ring vertices lie at the strand radius around the control point, normals radial
    off = pos - centres
    assert np.allclose(np.linalg.norm(off, axis=1), radii, rtol=1e-5, atol=1e-6)
    assert np.allclose(nrm * radii[:, None], off, atol=1e-5)
    # unit tangents, orthogonal to the radial direction
    assert np.allclose(np.linalg.norm(tan, axis=1), 1.0, atol=1e-5)
    assert np.abs((tan * nrm).sum(1)).max() < 1e-5
    # UV: position along the strand, (h + 1) / 2 with h = -cos(2 pi k / S)  (stored unflipped for hair)
    k = np.tile(np.arange(S), len(uv) // S)
    assert np.allclose(uv[:, 1], (1.0 - np.cos(2 * np.pi * k / S)) / 2, atol=1e-6)
    first = uv.reshape(-1, S, 2)[:, 0, 0]
    assert first.min() == 0.0 and first.max() == 1.0
    mats = (pt.pt_material * 1)()
    nori.nori_materials(h, mats, 1)
    assert mats[0].type == pt.PT_MAT_HAIR and abs(mats[0].roughness - 0.2) < 1e-7 and abs(mats[0].intIOR - 1.55) < 1e-7
    nori.nori_free(h)


@pytest.mark.parametrize("case,msg", [("signature", "not a HAIR file"), ("counts", "do not add up"),
                                      ("truncated", "truncated"), ("nopoints", "no points array")])
def test_hair_file_errors(nori, tmp_path, case, msg):
    s = wavy_strands(3, 4)
    p = tmp_path / "strands.hair"
    write_hair(p, s)
    b = bytearray(p.read_bytes())
    if case == "signature":
        b[0:4] = b"HAIX"
    elif case == "counts":  # first strand's segment count one short of its points
        b[128:130] = (int.from_bytes(b[128:130], "little") - 1).to_bytes(2, "little")
    elif case == "truncated":
        b = b[:200]
    elif case == "nopoints":
        b[12:16] = (int.from_bytes(b[12:16], "little") & ~2).to_bytes(4, "little")
    p.write_bytes(bytes(b))
    (tmp_path / "scene.xml").write_text(HAIR_XML.format(sides=6, scale=1.0))
    h, err = load(nori, tmp_path / "scene.xml")
    assert not h and msg in err, err


@pytest.mark.gpu
def test_hair_xml_furnace_matches_direct_scene(nori, pt, hair_dir):
    """The reference's hair white-furnace setup (white BCSDF colour, white
    envmap, path_mis) on a synthetic strand file: the XML render equals the
    same buffers rendered through libpt, and conserves energy to 3e-3."""
    d, _, _ = hair_dir
    h, err = load(nori, d / "scene.xml")
    assert h, err
    W, H = 64, 48
    s = np.zeros((H, W, 4), np.float32)
    c = np.zeros_like(s)
    st = pt.pt_stats()
    e = C.create_string_buffer(512)
    assert nori.nori_render(h, 64, 0, s.ctypes.data, c.ctypes.data, C.byref(st), e, 512) == 0, e.value
    mats = (pt.pt_material * 1)()
    nori.nori_materials(h, mats, 1)
    cam = pt.pt_camera()
    nori.nori_camera(h, C.byref(cam))
    pos, nrm, uv, tan, idx, env = (flat(nori, h, k) for k in range(6))
    ew = int(nori.nori_flat(h, 6, None))
    sc = pt.Scene(pos, idx, list(mats), normals=nrm, texcoords=uv, tangents=tan, env_rgb=env.reshape(-1, ew, 3))
    ctx = pt.Context(0)
    ctx.upload(sc)
    dd, _, _ = ctx.render(pt.render_params(W, H, 64, cam, max_depth=32))
    ctx.close()
    assert np.array_equal(s, dd), np.abs(s - dd).max()
    img = (s[..., :3] - c[..., :3]) / 64.0
    hairpix = img[np.abs(img - 1.0).max(-1) > 1e-6]
    assert len(hairpix) > 200  # the strands cover part of the frame
    assert abs(float(img.mean()) - 1.0) < 3e-3 and abs(float(hairpix.mean()) - 1.0) < 1e-2
    nori.nori_free(h)


def flat(nori, h, which):
    n = int(nori.nori_flat(h, which, None))
    a = np.zeros(n, np.uint32 if which == 4 else np.float32)
    nori.nori_flat(h, which, a.ctypes.data)
    return a


def scene_from_xml(nori, pt, path):
    """Load a Nori XML scene through the host (parser, plugins, OBJ loader,
    flattening, camera conversion) and rebuild the flattened arrays as a
    pt.Scene, so the oracle, the reference build and libpt all see the scene
    the host would upload.  Returns (scene, camera, info) with info as
    nori_info (width, height, spp, meshes, triangles, emitters, medium,
    max depth).  Scenes with textures or media are not rebuilt here."""
    h, err = load(nori, path)
    assert h, err
    try:
        info = (C.c_uint32 * 8)()
        nori.nori_info(h, info)
        assert info[6] == 0 and int(nori.nori_flat(h, 7, None)) == 0, "textures / media are not rebuilt"
        n = nori.nori_materials(h, None, 0)
        mats = (pt.pt_material * n)()
        nori.nori_materials(h, mats, n)
        cam = pt.pt_camera()
        nori.nori_camera(h, C.byref(cam))
        pos, nrm, uv, tan, idx, env = (flat(nori, h, k) for k in range(6))
        ew = int(nori.nori_flat(h, 6, None))
        sc = pt.Scene(pos, idx, list(mats), normals=nrm if nrm.size else None, texcoords=uv if uv.size else None,
                      tangents=tan if tan.size else None, env_rgb=env.reshape(-1, ew, 3),
                      env_scale=float(nori.nori_env_scale(h)))
        return sc, cam, list(info)
    finally:
        nori.nori_free(h)


SSS_XML = SCENE_XML.replace('''    <bsdf type="disney">
      <color name="baseColor" value="0.8, 0.3, 0.2"/>
      <float name="roughness" value="0.4"/><float name="metallic" value="0.2"/><float name="clearcoat" value="0.5"/>
    </bsdf>''', '''    <bsdf type="subsurface">
      <color name="albedo" value="0.9, 0.5, 0.4"/><float name="radius" value="0.1"/>
      <float name="intIOR" value="1.4"/><float name="extIOR" value="1.0"/><float name="g" value="0.3"/>
      <float name="roughness" value="0.25"/><color name="tint" value="1, 0.9, 0.8"/>
    </bsdf>''')


def test_subsurface_plugin_flattening(nori, pt, scene_dir):
    """The subsurface plugin maps radius / g / tint to the GPU record fields
    as the reference's getGPUData does (src/cpu/subsurface.cpp:69-89)."""
    (scene_dir / "sss.xml").write_text(SSS_XML)
    h, err = load(nori, scene_dir / "sss.xml")
    assert h, err
    mats = (pt.pt_material * 3)()
    nori.nori_materials(h, mats, 3)
    m = mats[0]
    assert m.type == pt.PT_MAT_SUBSURFACE
    assert np.allclose(list(m.albedo), [0.9, 0.5, 0.4]) and abs(m.subsurface - 0.1) < 1e-7
    assert abs(m.anisotropic - 0.3) < 1e-7 and abs(m.roughness - 0.25) < 1e-7
    assert np.allclose([m.sheen, m.sheenTint, m.clearcoat], [1.0, 0.9, 0.8])
    nori.nori_free(h)


@pytest.mark.gpu
def test_subsurface_xml_render_matches_direct_scene(nori, pt, scene_dir):
    (scene_dir / "sss.xml").write_text(SSS_XML)
    h, err = load(nori, scene_dir / "sss.xml")
    assert h, err
    W, H = 64, 48
    s = np.zeros((H, W, 4), np.float32)
    c = np.zeros_like(s)
    e = C.create_string_buffer(512)
    assert nori.nori_render(h, 4, 0, s.ctypes.data, c.ctypes.data, None, e, 512) == 0, e.value
    mats = (pt.pt_material * 3)()
    nori.nori_materials(h, mats, 3)
    cam = pt.pt_camera()
    nori.nori_camera(h, C.byref(cam))
    pos, nrm, uv, tan, idx, env = (flat(nori, h, k) for k in range(6))
    ew = int(nori.nori_flat(h, 6, None))
    sc = pt.Scene(pos, idx, list(mats), normals=nrm, texcoords=uv, tangents=tan, env_rgb=env.reshape(-1, ew, 3),
                  env_scale=0.5)
    ctx = pt.Context(0)
    ctx.upload(sc)
    d, _, _ = ctx.render(pt.render_params(W, H, 4, cam, max_depth=8))
    ctx.close()
    assert np.array_equal(s, d), np.abs(s - d).max()
    nori.nori_free(h)


def test_scene_files_resolve_per_scene(nori, pt, tmp_path):
    """Relative file names resolve against the scene's own directory: a scene
    loaded later in the same process does not pick up an earlier scene's
    files (here the default envmap textures/white_furnace.hdr)."""
    xml = """<scene><camera type="perspective"><integer name="width" value="8"/>
      <integer name="height" value="8"/></camera>
      <mesh type="obj"><string name="filename" value="tri.obj"/></mesh></scene>"""
    for name, with_env in (("a", True), ("b", False)):
        d = tmp_path / name
        (d / "textures").mkdir(parents=True)
        write_obj(d / "tri.obj", np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float), np.array([[0, 1, 2]]))
        if with_env:
            write_hdr(d / "textures" / "white_furnace.hdr", np.ones((2, 2, 3), np.float32))
        (d / "scene.xml").write_text(xml)
    sa, _, _ = scene_from_xml(nori, pt, tmp_path / "a" / "scene.xml")
    sb, _, _ = scene_from_xml(nori, pt, tmp_path / "b" / "scene.xml")
    sa2, _, _ = scene_from_xml(nori, pt, tmp_path / "a" / "scene.xml")
    assert np.array_equal(sa.env_rgb, np.ones((2, 2, 3), np.float32))
    assert np.array_equal(sb.env_rgb, np.full((1, 1, 3), 0.5, np.float32))
    assert np.array_equal(sa2.env_rgb, sa.env_rgb)
