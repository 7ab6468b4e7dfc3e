"""Whole renders through pt_render against the oracle, plus film semantics.

The wavefront integrator draws the same sample dimensions as RayGen, so at
one sample per pixel each pixel is one path that the oracle also traces;
paths leave each other only where float rounding flips a discrete choice
(lobe pick, Russian roulette, a hit near a triangle edge).
"""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "furnace.json")))


def relmse(x, ref):
    """validation_tests/compare_exr.py:101-103: mean((x - ref)^2 / (ref^2 + 1e-2))."""
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def mean_img(s):
    return s[..., :3] / np.maximum(s[..., 3:4], 1.0)


SCENES = {
    "cornell": (lambda sc: sc.cornell(64, 64), 64, 64, 8),
    "spheres": (lambda sc: sc.disney_spheres(80, 48, grid=3, slices=48, rings=25, env_w=256, env_h=128), 80, 48, 16),
    "hair_volume": (lambda sc: sc.hair_volume(48, 48, strands=300, segments=8, grid_n=32), 48, 48, 8),
}


@pytest.mark.parametrize("name", ["cornell", "spheres", "spheres_plan"])
def test_per_path_parity(name, pt, scenes, ctx, oracle):
    """Per-path equality with the oracle; spheres_plan renders over the 8-wide
    tree of the least-area plan (PT_DEBUG_WIDE_PLAN)."""
    plan = name.endswith("_plan")
    name = name.replace("_plan", "")
    make, W, H, depth = SCENES[name]
    sc, cam = make(scenes)
    ctx.debug_set(pt.PT_DEBUG_WIDE_PLAN, 1 if plan else 0)
    try:
        ctx.upload(sc)
    finally:
        ctx.debug_set(pt.PT_DEBUG_WIDE_PLAN, 0)
    oracle.load(sc)
    P = pt.render_params(W, H, 1, cam, max_depth=depth, sample_offset=3)
    sg, _, st = ctx.render(P)
    so, per, (o_ext, o_nee) = oracle.render(P, per_path=True)
    assert np.all(sg[..., 3] == 1.0)
    g, o = sg[..., :3], per[0]
    close = np.abs(g - o) <= 1e-3 * np.maximum(np.abs(o), 1e-2)
    frac = float(close.all(-1).mean())
    print(name, "pixels matching the oracle path:", frac, "rays", st.extension_rays, st.shadow_rays,
          "oracle", o_ext, o_nee)
    assert frac > 0.97, frac
    # The per-path ray counts of the bench's algorithmic bytes, checked against
    # the oracle: one closest-hit trace per bounce on both sides (equal up to
    # the few paths that differ); the oracle counts every NEE estimate, the
    # device only the shadow rays it traces (an estimate already zero is not
    # traced; the Cornell box's black envmap yields no envmap NEE rays), so
    # that count is at most the oracle's.
    assert abs(int(st.extension_rays) - int(o_ext)) <= 0.01 * o_ext, (st.extension_rays, o_ext)
    assert 0.2 * o_nee <= st.shadow_rays <= o_nee, (st.shadow_rays, o_nee)


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_image_relmse(name, pt, scenes, ctx, oracle):
    make, W, H, depth = SCENES[name]
    sc, cam = make(scenes)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(W, H, 16, cam, max_depth=depth)
    sg, _, _ = ctx.render(P)
    so, _, _ = oracle.render(P)
    r = relmse(mean_img(sg), mean_img(so))
    print(name, "relMSE(gpu, oracle) at 16 spp:", r)
    assert r < 1e-3, r


def test_volume_scene_statistical_parity(pt, scenes, ctx, oracle):
    """Media: the reference's null-collision walk steps exactly onto brick
    boundaries, where the brick chosen (and so the number of uniforms drawn)
    follows the last bit of the position; any rounding difference upstream
    (FMA, a 1-ulp transcendental) forks the path.  Parity is therefore
    statistical: at 256 spp the GPU image is as close to the oracle's as two
    oracle renders of disjoint samples are to each other."""
    make, W, H, depth = SCENES["hair_volume"]
    sc, cam = make(scenes)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(W, H, 256, cam, max_depth=depth)
    sg, _, _ = ctx.render(P)
    so, _, _ = oracle.render(P)
    sb, _, _ = oracle.render(pt.render_params(W, H, 256, cam, max_depth=depth, sample_offset=100000))
    g, o, b = mean_img(sg), mean_img(so), mean_img(sb)
    noise = relmse(b, o)
    r = relmse(g, o)
    print("hair_volume relMSE gpu-oracle", r, "oracle-oracle (disjoint samples)", noise)
    assert r < 2.0 * noise + 1e-4
    assert abs(float(g.mean()) / float(o.mean()) - 1.0) < 0.01
    _, per, _ = oracle.render(pt.render_params(W, H, 1, cam, max_depth=depth), per_path=True)
    s1, _, _ = ctx.render(pt.render_params(W, H, 1, cam, max_depth=depth))
    frac = float((np.abs(s1[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)).all(-1).mean())
    print("hair_volume pixels matching the oracle path:", frac)
    assert frac > 0.5


def test_deterministic_and_split_invariant(pt, scenes, ctx):
    sc, cam = scenes.cornell(48, 40)
    ctx.upload(sc)
    P = pt.render_params(48, 40, 4, cam, max_depth=8)
    a, ca, _ = ctx.render(P)
    b, cb, _ = ctx.render(P)
    assert np.array_equal(a, b) and np.array_equal(ca, cb)
    # the same samples in two calls (film carried through) or in small waves
    P1 = pt.render_params(48, 40, 2, cam, max_depth=8)
    P2 = pt.render_params(48, 40, 2, cam, max_depth=8, sample_offset=2)
    s, c, _ = ctx.render(P1)
    s, c, _ = ctx.render(P2, s, c)
    assert np.array_equal(a, s) and np.array_equal(ca, c)
    Pw = pt.render_params(48, 40, 4, cam, max_depth=8, wave_paths=999)
    w, cw, _ = ctx.render(Pw)
    assert np.array_equal(a, w)


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_graph_replay_matches_direct_launches(name, pt, scenes, ctx):
    """Renders replay a captured CUDA graph of their launches; with per-launch
    timing they issue the launches directly.  Same films, bit for bit, also
    when one graph is replayed with another sample offset."""
    make, W, H, depth = SCENES[name]
    sc, cam = make(scenes)
    ctx.upload(sc)
    for off in (0, 7, 1000):
        P = pt.render_params(W, H, 3, cam, max_depth=depth, sample_offset=off)
        Pt = pt.render_params(W, H, 3, cam, max_depth=depth, sample_offset=off, flags=pt.PT_RENDER_STAGE_TIMING)
        g, cg, sg = ctx.render(P)
        d, cd, sd = ctx.render(Pt)
        assert np.array_equal(g, d) and np.array_equal(cg, cd), off
        assert sg.extension_rays == sd.extension_rays and sg.launches == sd.launches
        assert sd.ms_extend > 0 and sg.ms_extend == 0


def test_pcg_sampler_parity(pt, scenes, ctx, oracle):
    sc, cam = scenes.cornell(48, 48)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(48, 48, 1, cam, max_depth=8, rng_kind=pt.PT_RNG_PCG_HASH)
    sg, _, _ = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    close = np.abs(sg[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)
    assert close.all(-1).mean() > 0.97


def test_alias_sampling_unbiased(pt, scenes, ctx):
    """Alias-table envmap sampling has the CDF's density: renders with either
    converge to the same image (smooth sky, so 256 spp is well converged)."""
    sc, cam = scenes.disney_spheres(64, 48, grid=2, slices=32, rings=17, env_w=256, env_h=128)
    sc.env_rgb[:] = scenes.sky_envmap(256, 128, sun_peak=30.0, sun_sigma_deg=6.0)
    ctx.upload(sc)
    a, _, _ = ctx.render(pt.render_params(64, 48, 256, cam, max_depth=16, env_sampling=pt.PT_ENV_CDF))
    b, _, _ = ctx.render(pt.render_params(64, 48, 256, cam, max_depth=16, env_sampling=pt.PT_ENV_ALIAS))
    ma, mb = mean_img(a), mean_img(b)
    assert abs(float(ma.mean()) / float(mb.mean()) - 1.0) < 0.005
    assert relmse(mb, ma) < 1e-3


@pytest.mark.parametrize("lobe", ["diffuse", "metallic_smooth", "metallic_rough", "clearcoat", "lambertian"])
def test_disney_furnace_gpu(lobe, pt, scenes, ctx):
    from test_oracle_golden import furnace_scene
    sc, cam, g = furnace_scene(pt, scenes, lobe)
    ctx.upload(sc)
    s, _, _ = ctx.render(pt.render_params(128, 128, 64, cam, max_depth=32))
    mean = float(mean_img(s).mean())
    assert abs(mean / g["mitsuba_image_mean"] - 1.0) < g["tolerance_rel"], (lobe, mean)


@pytest.mark.parametrize("name", ["beer_lambert", "white_furnace"])
def test_volume_golden_gpu(name, pt, scenes, ctx):
    from test_oracle_golden import volume_scene
    sc, cam, g = volume_scene(pt, scenes, name)
    ctx.upload(sc)
    s, _, _ = ctx.render(pt.render_params(64, 64, 256, cam, max_depth=32))
    mean = float(mean_img(s).mean())
    assert abs(mean - g["expected"]) < g["tolerance_abs"], (name, mean)


def test_hair_white_furnace_gpu(pt, ctx, oracle):
    """The GPU hair BCSDF integrates to the same energy as the oracle's."""
    from test_oracle_golden import hair_furnace_integral

    class GpuEval:
        def bsdf_eval(self, mats, mi, wi, wo, h, fp64=False):
            return ctx.bsdf_eval(mats, mi, wi, wo, h)

    for h in (-0.6, 0.0, 0.7):
        eg = hair_furnace_integral(pt, GpuEval(), h)
        eo = hair_furnace_integral(pt, oracle, h)
        assert abs(eg - eo) < 1e-4 and abs(eg - 1.0) < 3e-3, (h, eg, eo)


def test_heterogeneous_media_wavefront(pt, scenes, ctx, oracle):
    """PT_RENDER_MEDIA_WAVEFRONT runs heterogeneous media in the wavefront
    form (deferred NEE, ratio tracking drawn before visibility): the same
    estimator with another order of draws, so parity with the oracle is
    statistical as for the inline form; and it is faster."""
    make, W, H, depth = SCENES["hair_volume"]
    sc, cam = make(scenes)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(W, H, 256, cam, max_depth=depth, flags=pt.PT_RENDER_MEDIA_WAVEFRONT)
    sg, _, st = ctx.render(P)
    so, _, _ = oracle.render(pt.render_params(W, H, 256, cam, max_depth=depth))
    sb, _, _ = oracle.render(pt.render_params(W, H, 256, cam, max_depth=depth, sample_offset=100000))
    g, o, b = mean_img(sg), mean_img(so), mean_img(sb)
    noise = relmse(b, o)
    r = relmse(g, o)
    print("hair_volume wavefront relMSE gpu-oracle", r, "oracle-oracle", noise)
    assert r < 2.0 * noise + 1e-4
    assert abs(float(g.mean()) / float(o.mean()) - 1.0) < 0.01
    # same requests in a batch with the flag: identical films
    reqs = [pt.render_params(W, H, 2, cam, max_depth=depth, flags=pt.PT_RENDER_MEDIA_WAVEFRONT),
            pt.render_params(32, 24, 3, cam, max_depth=depth, sample_offset=7, flags=pt.PT_RENDER_MEDIA_WAVEFRONT)]
    films, _, _ = ctx.render_batch(reqs)
    for Q, (s, c) in zip(reqs, films):
        s1, c1, _ = ctx.render(Q)
        assert np.array_equal(s, s1) and np.array_equal(c, c1)


@pytest.mark.parametrize("name", ["cornell", "spheres", "cool_scene1", "textured", "subsurface"])
def test_tail_kernel_leaves_no_trace(name, pt, scenes):
    """From bounce 4 on, a wave with at most 2^17 live paths and at least 8
    bounces left runs its paths to the end in one kernel; otherwise it stays
    in the per-bounce kernels.  Both run the same shading code per path (the
    class-specialized kernels' code with NEE resolved as the shadow kernel
    does, or the inline form for subsurface scenes), so the film may not
    depend on which ran: the same render with the tail and, through the
    PT_DEBUG_TAIL hook, without it, equal bit for bit (and the tail checked
    to have traced rays).  At depth 8 the default rule keeps the per-bounce
    kernels, and mode 2 forces the tail: again the same film.  The classes
    covered: miss, emitter, diffuse, Disney (Cornell, spheres), delta
    (mirror and glass), textured Disney and diffuse with an alpha cut-out,
    and the inline form (subsurface)."""
    if name == "cornell":
        sc, cam = scenes.cornell(128, 128)
        W = H = 128
    elif name == "spheres":
        sc, cam = scenes.disney_spheres(160, 90, grid=4, slices=32, rings=17, env_w=256, env_h=128)
        W, H = 160, 90
    elif name == "cool_scene1":
        from test_reference_scenes import load_scene
        sc, cam, _ = load_scene(pt, "cool_scene1")
        W = H = 128
    elif name == "textured":
        sc, cam = scenes.textured_scene(128, 96)
        W, H = 128, 96
    else:
        sc, cam = scenes.subsurface_scene(128, 128)
        W = H = 128
    ctx = pt.Context(0)
    try:
        ctx.upload(sc)
        P = pt.render_params(W, H, 16, cam, max_depth=16, sample_offset=5)
        a, ca, sa = ctx.render(P)
        ctx.debug_set(pt.PT_DEBUG_TAIL, 1)
        b, cb, sb = ctx.render(P)
        ctx.debug_set(pt.PT_DEBUG_TAIL, 0)
        c, cc, sc2 = ctx.render(P)
        P8 = pt.render_params(W, H, 16, cam, max_depth=8, sample_offset=5)
        d, cd, sd = ctx.render(P8)
        ctx.debug_set(pt.PT_DEBUG_TAIL, 2)
        e, ce, se = ctx.render(P8)
        ctx.debug_set(pt.PT_DEBUG_TAIL, 0)
    finally:
        ctx.close()
    assert sd.tail_extension_rays == 0 and se.tail_extension_rays > 0
    assert np.array_equal(d, e) and np.array_equal(cd, ce)
    print(name, "tail extension rays", sa.tail_extension_rays, "of", sa.extension_rays)
    assert sa.tail_extension_rays > 0 and sb.tail_extension_rays == 0 and sc2.tail_extension_rays > 0
    assert sa.extension_rays == sb.extension_rays and sa.shadow_rays == sb.shadow_rays
    assert np.array_equal(a, b) and np.array_equal(ca, cb)
    assert np.array_equal(a, c)
