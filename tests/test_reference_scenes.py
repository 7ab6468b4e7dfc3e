"""The reference's own scenes and validation images.

Scenes are the reference's XML files loaded unmodified through the Nori host
(parser, plugin registry, OBJ loader, flattening, camera conversion); the
flattened arrays are kept in tests/golden/scenes (tests/golden/
make_scene_fixtures.py) because the reference checkout is not present where
the GPU tests run, and are re-derived from the XML here whenever it is:

* scenes/cool_scene1/cornell_box.xml — the reference's demo box: diffuse
  walls, a mirror sphere, a glass sphere and a quad light.  Its envmap
  (sunset.hdr) is not in the checkout, so the host falls back to a grey
  texel as the reference does (DXRApp_Textures.cpp:181-210), at the scene's
  envmapScale 0.  No integrator is named: the reference's GPU build always
  runs its path tracer (32 bounces), and so does the host.
* validation_tests/dof/dof_test_scene.xml (thin lens: radius 0.1, focal
  distance 4) and dof_pinhole_scene.xml (the same with radius 0).
* validation_tests/disney/furnace_*.xml and
  validation_tests/ibl_test/sphere_furnace_ibl.xml — white furnaces.

Checks: the oracle gives the reference build's bits on these scenes (CPU);
the GPU follows the oracle path by path (mirror, glass, glass shadow rays,
thin-lens raygen); whole GPU images match the reference's own GPU renders
of the validation scenes (diff_*/ours_srgb.png, tonemapped 8 bit) and the
Mitsuba furnace images, per pixel (GPU)."""

import ctypes as C
import os

import numpy as np
import pytest

from test_nori_host import nori, scene_from_xml  # noqa: F401  (nori: fixture)

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_scene(pt, name):
    """(pt.Scene, camera, info) rebuilt from tests/golden/scenes/<name>.npz."""
    z = np.load(os.path.join(GOLDEN, "scenes", name + ".npz"))
    nm = len(z["materials"]) // C.sizeof(pt.pt_material)
    mats = (pt.pt_material * nm).from_buffer_copy(z["materials"].tobytes())
    cam = pt.pt_camera.from_buffer_copy(z["camera"].tobytes())

    def opt(k):
        return z[k] if z[k].size else None

    sc = pt.Scene(z["positions"], z["indices"], list(mats), normals=opt("normals"), texcoords=opt("texcoords"),
                  tangents=opt("tangents"), env_rgb=z["env_rgb"], env_scale=float(z["env_scale"]))
    return sc, cam, [int(x) for x in z["info"]]


def reference_file(rel):
    from oracle.oracle import REF_ROOT

    p = os.path.join(REF_ROOT, rel)
    if not os.path.exists(p):
        pytest.skip("reference checkout not present")
    return p


def tonemap8(img):
    """The reference comparison tool's display curve (validation_tests/
    compare_exr.py:57-62: x/(1+x), then x^(1/2.2)) on a 0..255 scale."""
    x = np.maximum(img.astype(np.float64), 0.0)
    return np.power(x / (1.0 + x), 1.0 / 2.2) * 255.0


def relmse(x, ref):
    """validation_tests/compare_exr.py:101-103."""
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


SCENE_NAMES = ["cool_scene1", "dof", "dof_pinhole", "furnace_ibl", "furnace_diffuse", "furnace_metallic_smooth",
               "furnace_metallic_rough", "furnace_clearcoat", "furnace_lambertian"]


@pytest.mark.parametrize("name", SCENE_NAMES)
def test_fixture_matches_the_xml(name, pt, nori):  # noqa: F811
    """The committed arrays are what the host makes of the XML today."""
    z = np.load(os.path.join(GOLDEN, "scenes", name + ".npz"))
    sc, cam, info = scene_from_xml(nori, pt, reference_file(str(z["source"])))
    assert np.array_equal(sc.positions, z["positions"]) and np.array_equal(sc.indices, z["indices"])
    assert bytes(sc.materials) == z["materials"].tobytes() and bytes(cam) == z["camera"].tobytes()
    assert np.array_equal(sc.env_rgb, z["env_rgb"]) and sc.env_scale == float(z["env_scale"])
    assert list(info) == [int(x) for x in z["info"]]
    for k, a in (("normals", sc.normals), ("texcoords", sc.texcoords), ("tangents", sc.tangents)):
        assert np.array_equal(np.zeros(0, np.float32) if a is None else a, z[k]), k


def test_cool_scene1_as_the_reference_sees_it(pt):
    """Six meshes: three diffuse walls, a mirror, a dielectric (the BK7 /
    air defaults of src/cpu/dielectric.cpp) and the light; the missing
    sunset.hdr becomes one grey texel at envmapScale 0; 800 x 800; the
    default GPU integrator with 32 bounces."""
    sc, cam, info = load_scene(pt, "cool_scene1")
    types = [m.type for m in sc.materials]
    assert types == [pt.PT_MAT_DIFFUSE] * 3 + [pt.PT_MAT_MIRROR, pt.PT_MAT_DIELECTRIC, pt.PT_MAT_DIFFUSE]
    glass = sc.materials[4]
    assert abs(glass.intIOR - 1.5046) < 1e-6 and abs(glass.extIOR - 1.000277) < 1e-6
    assert np.array_equal(sc.env_rgb, np.full((1, 1, 3), 0.5, np.float32)) and sc.env_scale == 0.0
    assert info[:2] == [800, 800] and info[5] == 1 and info[7] == 32
    assert cam.lens_radius == 0.0


def test_dof_camera(pt):
    _, cam, info = load_scene(pt, "dof")
    assert abs(cam.lens_radius - 0.1) < 1e-7 and abs(cam.focal_distance - 4.0) < 1e-6
    _, cam0, _ = load_scene(pt, "dof_pinhole")
    assert cam0.lens_radius == 0.0
    assert info[:3] == [512, 512, 256]


@pytest.mark.parametrize("name,W,spp", [("cool_scene1", 96, 8), ("dof", 64, 8)])
def test_oracle_is_the_reference_build(name, W, spp, pt, oracle, reference):
    """Mirror and glass shading, glass shadow rays and the thin-lens camera:
    the oracle gives the reference build's image bit for bit."""
    sc, cam, _ = load_scene(pt, name)
    oracle.load(sc)
    reference.load(sc)
    P = pt.render_params(W, W, spp, cam, max_depth=32, sample_offset=7)
    so, _, _ = oracle.render(P, threads=4)
    sr = reference.render(P, threads=4)
    assert np.array_equal(so, sr)
    assert so[..., 3].min() == spp


# ---- GPU -----------------------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name,W", [("cool_scene1", 128), ("dof", 128), ("dof_pinhole", 96)])
def test_per_path_parity(name, W, pt, ctx, oracle):
    """One sample per pixel is one path that the oracle also traces: mirror
    reflections, glass refraction with its Fresnel draw, NEE through the
    glass sphere ((1 - Fr) per glass crossing), thin-lens rays."""
    sc, cam, _ = load_scene(pt, name)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(W, W, 1, cam, max_depth=32, sample_offset=3)
    sg, _, st = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    g, o = sg[..., :3], per[0]
    frac = float((np.abs(g - o) <= 1e-3 * np.maximum(np.abs(o), 1e-2)).all(-1).mean())
    print(name, "pixels matching the oracle path:", frac, "rays", st.extension_rays, st.shadow_rays)
    assert frac > 0.97, frac
    P16 = pt.render_params(W, W, 16, cam, max_depth=32, sample_offset=11)
    s16, _, _ = ctx.render(P16)
    o16, _, _ = oracle.render(P16)
    r = relmse(s16[..., :3] / s16[..., 3:4], o16[..., :3] / o16[..., 3:4])
    print(name, "relMSE(gpu, oracle) at 16 spp:", r)
    assert r < 1e-3, r


def _gpu_image(pt, ctx, name, spp=None, offset=0):
    sc, cam, info = load_scene(pt, name)
    ctx.upload(sc)
    W, H = info[0], info[1]
    # the reference's GPU build runs its path tracer (32 bounces) whatever
    # integrator the XML names
    s, _, _ = ctx.render(pt.render_params(W, H, spp or info[2], cam, max_depth=32, sample_offset=offset))
    return s[..., :3] / s[..., 3:4]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["dof", "dof_pinhole", "furnace_ibl", "furnace_diffuse", "furnace_metallic_smooth",
                                  "furnace_metallic_rough", "furnace_clearcoat"])
def test_matches_the_reference_gpu_render(name, pt, ctx):
    """The GPU image at the XML's resolution and spp against the reference's
    own GPU render of the same XML (its comparison tool's ours_srgb.png),
    per pixel after the same tonemap: the difference is the two renders'
    noise (8-bit, unbiased).  For the depth-of-field pair the golden is 2x2
    block means, and swapping lens and pinhole fails these bounds (p99 ~80,
    5 % of blocks beyond 8)."""
    img = _gpu_image(pt, ctx, name)
    g = np.load(os.path.join(GOLDEN, "images", name + ".npz"))
    b = int(g["dxr_binned"])
    t8 = tonemap8(img)
    if b > 1:
        H, W = t8.shape[:2]
        t8 = t8.reshape(H // b, b, W // b, b, 3).mean((1, 3))
    d = t8 - g["dxr_srgb"].astype(np.float64)
    st = {"mean_abs": float(np.abs(d).mean()), "bias": float(d.mean()), "p99": float(np.percentile(np.abs(d), 99)),
          "frac_gt8": float((np.abs(d) > 8).mean())}
    print(name, st)
    assert st["mean_abs"] < 1.6 and abs(st["bias"]) < 0.5 and st["p99"] < 12.0 and st["frac_gt8"] < 0.015, st


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["furnace_ibl", "furnace_diffuse", "furnace_metallic_smooth", "furnace_metallic_rough",
                                  "furnace_clearcoat", "furnace_lambertian"])
def test_matches_the_mitsuba_furnace(name, pt, ctx):
    """The reference's validation as written: the XML rendered at its
    resolution and spp, compared per pixel with the Mitsuba 3 image through
    the comparison tool's statistics (RMSE, relMSE) and the 2 % band on the
    mean of validation_tests/disney/README.md:68-72.  Bounds: the oracle's
    own figures on these scenes with room for noise (RMSE 0.002-0.025,
    relMSE <= 4.1e-4 except clearcoat, whose 0.042 is the reference's own
    disagreement with Mitsuba on the clearcoat lobe)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "pbrt_b200_compare", os.path.join(os.path.dirname(HERE), "pbrt-renderer-_b200", "compare.py"))
    cmp_ = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cmp_)
    img = _gpu_image(pt, ctx, name)
    ref = np.load(os.path.join(GOLDEN, "images", name + ".npz"))["mitsuba"].astype(np.float32)
    r = cmp_.compare(img, ref)
    ratio = r["ours_mean"] / r["ref_mean"]
    print(name, "rmse", r["rmse"], "relmse", r["relmse"], "mean ratio", ratio)
    assert abs(ratio - 1.0) < 0.02
    assert r["rmse"] < 0.04
    assert r["relmse"] < (0.06 if name == "furnace_clearcoat" else 1e-3)


@pytest.mark.gpu
def test_glass_shadow_transmission(pt, scenes, ctx, oracle):
    """Shadow rays through stacked glass and mirror panes
    (TraceShadowInline, shaders/RayQueryTrace.hlsli:88-129): glass never
    occludes, each crossing multiplies the transmission by 1 - Fr at the
    geometric normal; an opaque pane occludes.  GPU vs oracle per ray."""
    rng = np.random.default_rng(61)
    b = scenes._Builder()
    for k in range(7):  # panes at y = 0.5 .. 3.5, tilted, glass / mirror / one opaque
        y = 0.5 + 0.5 * k
        tilt = rng.uniform(-0.4, 0.4, 2)
        quad = np.array([[-2, y + tilt[0], -2], [2, y + tilt[1], -2], [2, y - tilt[0], 2], [-2, y - tilt[1], 2]],
                        np.float32)
        if k == 5:
            quad[:, 0] = quad[:, 0] * 0.3 + 1.2  # a narrow opaque strip
        kind = pt.PT_MAT_DIFFUSE if k == 5 else (pt.PT_MAT_MIRROR if k == 3 else pt.PT_MAT_DIELECTRIC)
        m = pt.make_material(kind, (0.8, 0.8, 0.8))
        m.intIOR, m.extIOR = float(rng.uniform(1.2, 2.2)), float(rng.uniform(1.0, 1.3))
        b.add(quad, [[0, 1, 2], [0, 2, 3]], m)
    sc = b.scene()
    ctx.upload(sc)
    oracle.load(sc)
    n = 200000
    o = np.stack([rng.uniform(-1.5, 1.5, n), np.zeros(n), rng.uniform(-1.5, 1.5, n)], -1).astype(np.float32)
    tgt = np.stack([rng.uniform(-1.5, 1.5, n), np.full(n, 4.5), rng.uniform(-1.5, 1.5, n)], -1).astype(np.float32)
    d = tgt - o
    dist = np.linalg.norm(d, axis=1)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7], rays[:, 7] = o, 1e-3, d / dist[:, None], dist
    occ_g, tr_g = ctx.trace_shadow(rays)
    occ_o, tr_o = oracle.trace_shadow(rays)
    assert np.array_equal(occ_g, occ_o)
    free = occ_o == 0
    assert free.mean() > 0.5 and (occ_o == 1).mean() > 0.05
    tg, to = tr_g[free], tr_o[free]
    assert (to < 0.99).all()  # every unoccluded ray crossed glass
    rel = np.abs(tg - to) / to
    print("transmission rel. difference: max", rel.max(), "p99.9", np.quantile(rel, 0.999))
    assert rel.max() < 1e-5
