"""The oracle restatement against the reference's own shader code.

oracle/build_ref.py compiles the reference's shaders (shaders/*.hlsl(i)) for
the CPU; these tests require the restatement in oracle/pt_oracle.cpp to give
the same bits for the scene buffers, the sample stream, the BSDFs, the envmap
tables and whole rendered images.
"""

import numpy as np
import pytest


def _scenes(scenes):
    return {
        "cornell": scenes.cornell(48, 40),
        "spheres": scenes.disney_spheres(40, 32, grid=2, slices=24, rings=13, env_w=128, env_h=64),
        "hair_volume": scenes.hair_volume(40, 40, strands=120, segments=6, grid_n=24),
        "subsurface": scenes.subsurface_scene(48, 40),
    }


@pytest.fixture(scope="module")
def scene_set(scenes):
    return _scenes(scenes)


@pytest.mark.parametrize("name", ["cornell", "spheres", "hair_volume"])
def test_scene_buffers_identical(name, scene_set, oracle, reference):
    sc, _ = scene_set[name]
    oracle.load(sc)
    reference.load(sc)
    assert bytes(oracle.materials()) == bytes(reference.materials())
    mo, co = oracle.env_cdf()
    mr, cr = reference.env_cdf()
    assert np.array_equal(mo, mr) and np.array_equal(co, cr)


def test_sample_stream_identical(oracle, reference):
    rng = np.random.default_rng(3)
    pix = rng.integers(0, 1 << 20, 4000).astype(np.uint32)
    smp = rng.integers(0, 4096, 4000).astype(np.uint32)
    a = oracle.rng(0, pix, smp, 24, 1024, 1024)
    b = reference.rng(pix, smp, 24, 1024, 1024)
    assert np.array_equal(a, b)


def test_bsdf_eval_identical(pt, scenes, oracle, reference):
    rng = np.random.default_rng(5)
    mats = []
    for t in (pt.PT_MAT_DIFFUSE, pt.PT_MAT_MICROFACET, pt.PT_MAT_DISNEY, pt.PT_MAT_HAIR, pt.PT_MAT_SUBSURFACE):
        for _ in range(4):
            m = pt.make_material(t, tuple(rng.uniform(0.05, 1, 3)))
            m.roughness, m.metallic, m.specular = rng.uniform(0.05, 1), rng.uniform(), rng.uniform()
            m.specularTint, m.sheen, m.sheenTint = rng.uniform(), rng.uniform(), rng.uniform()
            m.subsurface, m.clearcoat, m.clearcoatGloss = rng.uniform(), rng.uniform(), rng.uniform()
            m.alpha = rng.uniform(0.05, 0.8) if t == pt.PT_MAT_MICROFACET else 2.0
            if t == pt.PT_MAT_HAIR:
                m.roughness, m.betaN, m.intIOR = 0.3, 0.3, 1.55
            mats.append(m)
    n = 40000
    wi = scenes.sample_directions(n, 11)
    wo = scenes.sample_directions(n, 12)
    mi = (np.arange(n) % len(mats)).astype(np.uint32)
    h = rng.uniform(-1, 1, n).astype(np.float32)
    fo, po = oracle.bsdf_eval(mats, mi, wi, wo, h)
    fr, pr = reference.bsdf_eval(mats, mi, wi, wo, h)
    assert np.array_equal(fo, fr) and np.array_equal(po, pr)
    # MaterialSample: the reference draws from the path sampler; feed the
    # oracle the same draws.
    pix = np.arange(n, dtype=np.uint32) % (64 * 64)
    smp = (np.arange(n) // (64 * 64)).astype(np.uint32)
    u = oracle.rng(0, pix, smp, 4, 64, 64)
    wo_o, wt_o, p_o = oracle.bsdf_sample(mats, mi, wi, u, h)
    wo_r, wt_r, p_r = reference.bsdf_sample(mats, mi, wi, h, pix, smp, 0, 64, 64)
    assert np.array_equal(wo_o, wo_r) and np.array_equal(wt_o, wt_r) and np.array_equal(p_o, p_r)


def test_envmap_sample_identical(scene_set, oracle, reference):
    sc, _ = scene_set["spheres"]
    oracle.load(sc)
    reference.load(sc)
    u = np.random.default_rng(7).uniform(0, 1, (20000, 2)).astype(np.float32)
    do, ro, po = oracle.env_sample(0, u)
    dr, rr, pr = reference.env_sample(u)
    assert np.array_equal(do, dr) and np.array_equal(ro, rr) and np.array_equal(po, pr)
    po2, ro2 = oracle.env_pdf(0, do)
    pr2, rr2 = reference.env_pdf(do)
    assert np.array_equal(po2, pr2) and np.array_equal(ro2, rr2)


@pytest.mark.parametrize("name,depth", [("cornell", 8), ("spheres", 16), ("hair_volume", 8), ("subsurface", 8)])
def test_render_identical(name, depth, scene_set, pt, oracle, reference):
    sc, cam = scene_set[name]
    oracle.load(sc)
    reference.load(sc)
    W = 48 if name in ("cornell", "subsurface") else 40
    H = 40 if name != "spheres" else 32
    P = pt.render_params(W, H, 3, cam, max_depth=depth, sample_offset=5)
    so, _, _ = oracle.render(P, threads=4)
    sr = reference.render(P, threads=4)
    assert np.array_equal(so, sr)
    assert so[..., 3].min() == 3.0


@pytest.fixture(scope="module")
def reference_ris(pt):
    from oracle.oracle import Reference
    if not Reference.available(ris=True):
        pytest.skip("reference shader build with USE_RIS=1 (oracle/_ref/libref_ris.so) not present")
    return Reference(pt, ris=True)


@pytest.mark.parametrize("name", ["many_lights", "spheres"])
def test_ris_render_identical(name, scenes, pt, oracle, reference_ris):
    """PT_RENDER_RIS_NEE restates the reference's USE_RIS=1 build
    (RISDirectIllumination, shaders/Emitter.hlsli:155-271): same image bits."""
    if name == "many_lights":
        sc, cam = scenes.cornell(48, 40, many_lights=True)
        W, H, depth = 48, 40, 8
    else:
        sc, cam = scenes.disney_spheres(40, 32, grid=2, slices=24, rings=13, env_w=128, env_h=64)
        W, H, depth = 40, 32, 16
    oracle.load(sc)
    reference_ris.load(sc)
    P = pt.render_params(W, H, 3, cam, max_depth=depth, sample_offset=2, flags=pt.PT_RENDER_RIS_NEE)
    so, _, _ = oracle.render(P, threads=4)
    sr = reference_ris.render(P, threads=4)
    assert np.array_equal(so, sr)
    # with area lights RIS draws other samples than MIS (without any it is MIS)
    P2 = pt.render_params(W, H, 3, cam, max_depth=depth, sample_offset=2)
    sm, _, _ = oracle.render(P2, threads=4)
    assert np.array_equal(so, sm) == (name == "spheres")
