"""libpt (CUDA, through the C ABI) against the CPU oracle.

Integer work (sample stream, Morton codes, radix-tree topology, envmap CDF
tables) must be bit-exact.  Float work is compared per element against the
oracle's float32 result, with the error of both stated against the oracle's
FP64 evaluation, on 1M seeded direction pairs per material type:

* relative difference GPU vs float32 oracle <= 1e-5 for >= 99 % of pairs and,
  for >= 99.9 %, <= 5e-5 or the oracle's own 99.9th-percentile error against
  FP64 where that is larger (floor 1e-6 of the median magnitude);
* the GPU is never less accurate than the float32 oracle: its error against
  FP64 is within 4x the oracle's own error + 1e-5 relative for >= 99.9 % of
  pairs, its 99.9th-percentile error against FP64 is at most 1.25x the
  oracle's, and its 99.99th-percentile and largest errors against FP64 at
  most 2x the oracle's.

Cancellation in the reference formulas (e.g. pow(1 - cos, 5), GTR1 at low
gloss) puts the float32 oracle itself ~2e-5 from FP64 at the 99.9th
percentile for the Disney BSDF, which is why the 1e-5 bar is stated at p99.
BSDF *sampling* maps uniforms to a direction first; near-delta lobes amplify
direction rounding into the value, so sampling is checked as (a) direction
parity against FP64 and (b) value parity at the GPU's own direction.
"""

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

N_PAIRS = 1 << 20


def random_materials(pt, rng, kind, count):
    mats = []
    for _ in range(count):
        m = pt.make_material(kind, tuple(rng.uniform(0.05, 1.0, 3)))
        if kind == pt.PT_MAT_DISNEY:
            m.roughness = rng.uniform(0.05, 1.0)
            m.metallic, m.specular, m.specularTint = rng.uniform(0, 1, 3)
            m.sheen, m.sheenTint, m.subsurface = rng.uniform(0, 1, 3)
            m.clearcoat, m.clearcoatGloss = rng.uniform(0, 1, 2)
        elif kind == pt.PT_MAT_MICROFACET:
            m.alpha = rng.uniform(0.05, 0.8)
        elif kind == pt.PT_MAT_HAIR:
            m.roughness, m.betaN = rng.uniform(0.2, 0.6), rng.uniform(0.2, 0.6)
            m.alpha, m.intIOR = 2.0, 1.55
        elif kind == pt.PT_MAT_SUBSURFACE:
            m.roughness, m.intIOR, m.extIOR = rng.uniform(0.05, 1.0), rng.uniform(1.2, 1.7), 1.0
        mats.append(m)
    return mats


def parity_stats(gpu, o32, o64, floor):
    d = rel_err(gpu, o32, floor)
    e_gpu = np.abs(gpu.astype(np.float64) - o64)
    e_or = np.abs(o32.astype(np.float64) - o64)
    bound = 4.0 * e_or + 1e-5 * np.maximum(np.abs(o64), floor)
    rg = e_gpu / np.maximum(np.abs(o64), floor)
    ro = e_or / np.maximum(np.abs(o64), floor)
    return {"p99": float(np.quantile(d, 0.99)), "p999": float(np.quantile(d, 0.999)),
            "p9999": float(np.quantile(d, 0.9999)), "max": float(d.max()),
            "frac_within_bound": float((e_gpu <= bound).mean()),
            "gpu_vs_fp64_p99": float(np.quantile(rg, 0.99)), "oracle_vs_fp64_p99": float(np.quantile(ro, 0.99)),
            "gpu_vs_fp64_p999": float(np.quantile(rg, 0.999)), "oracle_vs_fp64_p999": float(np.quantile(ro, 0.999)),
            "gpu_vs_fp64_p9999": float(np.quantile(rg, 0.9999)),
            "oracle_vs_fp64_p9999": float(np.quantile(ro, 0.9999)),
            "gpu_vs_fp64_max": float(rg.max()), "oracle_vs_fp64_max": float(ro.max())}


def assert_tail(st):
    """The worst pairs: a float32 evaluation of these formulas can itself be
    far from FP64 on a few pairs (cancellation), so the tail is bounded by
    the oracle's own: the GPU's 99.99th-percentile and worst errors against
    FP64 at most twice the oracle's."""
    assert st["gpu_vs_fp64_p9999"] <= 2.0 * st["oracle_vs_fp64_p9999"] + 1e-6, st
    assert st["gpu_vs_fp64_max"] <= 2.0 * st["oracle_vs_fp64_max"] + 1e-6, st


def assert_parity(st, accuracy_factor=1.25):
    # at the 99.9th percentile a difference below the float32 oracle's own
    # error against FP64 cannot be told apart from the oracle's rounding
    assert st["p99"] <= 1e-5 and st["p999"] <= max(5e-5, st["oracle_vs_fp64_p999"]), st
    assert st["frac_within_bound"] >= 0.999, st
    assert st["gpu_vs_fp64_p999"] <= accuracy_factor * st["oracle_vs_fp64_p999"] + 1e-6, st
    assert_tail(st)


def assert_parity_ill_conditioned(st):
    """For quantities whose float32 evaluation is itself far from FP64 (the
    pdf at a sampled direction of a near-specular GGX lobe: with alpha^2 ~ 6e-6
    one ulp of cos(theta_h) moves D by ~2 %): the GPU and the oracle err
    independently, so they may differ by up to twice the oracle's own error,
    and the GPU must be as accurate as the oracle against FP64 at p99 and
    p99.9.  Where the oracle's error is below the fixed bounds, those apply."""
    assert st["p99"] <= max(1e-5, 2 * st["oracle_vs_fp64_p99"]), st
    assert st["p999"] <= max(5e-5, 2 * st["oracle_vs_fp64_p999"]), st
    assert st["gpu_vs_fp64_p99"] <= 1.25 * st["oracle_vs_fp64_p99"] + 1e-6, st
    assert st["gpu_vs_fp64_p999"] <= 1.25 * st["oracle_vs_fp64_p999"] + 1e-6, st
    assert_tail(st)


def test_sample_stream_bit_exact(ctx, oracle):
    rng = np.random.default_rng(1)
    pix = rng.integers(0, 1280 * 720, 200000).astype(np.uint32)
    smp = rng.integers(0, 1 << 16, 200000).astype(np.uint32)
    for kind in (0, 1):
        a = ctx.rng(kind, pix, smp, 16, 1280, 720)
        b = oracle.rng(kind, pix, smp, 16, 1280, 720)
        assert np.array_equal(a, b), kind


@pytest.mark.parametrize("kind_name", ["DIFFUSE", "MICROFACET", "DISNEY", "HAIR", "SUBSURFACE"])
def test_bsdf_eval_parity(kind_name, pt, scenes, ctx, oracle):
    kind = getattr(pt, "PT_MAT_" + kind_name)
    rng = np.random.default_rng(17)
    mats = random_materials(pt, rng, kind, 64)
    wi = scenes.sample_directions(N_PAIRS, 21, upper=kind != pt.PT_MAT_HAIR)
    wo = scenes.sample_directions(N_PAIRS, 22, upper=kind != pt.PT_MAT_HAIR)
    mi = rng.integers(0, len(mats), N_PAIRS).astype(np.uint32)
    h = rng.uniform(-0.95, 0.95, N_PAIRS).astype(np.float32)
    fg, pg = ctx.bsdf_eval(mats, mi, wi, wo, h)
    f32, p32 = oracle.bsdf_eval(mats, mi, wi, wo, h)
    f64, p64 = oracle.bsdf_eval(mats, mi, wi, wo, h, fp64=True)
    scale_f = float(np.quantile(np.abs(f64), 0.5)) + 1e-12
    scale_p = float(np.quantile(np.abs(p64), 0.5)) + 1e-12
    sf = parity_stats(fg, f32, f64, 1e-6 * scale_f)
    sp = parity_stats(pg, p32, p64, 1e-6 * scale_p)
    print(kind_name, "f", sf, "pdf", sp)
    assert_parity(sf)
    assert_parity(sp)


@pytest.mark.parametrize("kind_name", ["DIFFUSE", "MICROFACET", "DISNEY", "HAIR"])
def test_bsdf_sample_parity(kind_name, pt, scenes, ctx, oracle):
    kind = getattr(pt, "PT_MAT_" + kind_name)
    rng = np.random.default_rng(29)
    mats = random_materials(pt, rng, kind, 64)
    n = N_PAIRS
    wi = scenes.sample_directions(n, 31, upper=kind != pt.PT_MAT_HAIR)
    u = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    mi = rng.integers(0, len(mats), n).astype(np.uint32)
    h = rng.uniform(-0.95, 0.95, n).astype(np.float32)
    wog, wtg, pg = ctx.bsdf_sample(mats, mi, wi, u, h)
    wo32, _, _ = oracle.bsdf_sample(mats, mi, wi, u, h)
    wo64, _, _ = oracle.bsdf_sample(mats, mi, wi, u, h, fp64=True)
    # (a) directions: the GPU's distance to the FP64 direction vs the oracle's
    valid = (pg > 0) & np.isfinite(wo64).all(1)
    e_gpu = np.abs(wog - wo64).max(1)
    e_or = np.abs(wo32 - wo64).max(1)
    same_lobe = e_gpu < 1e-2  # a lobe/branch pick flipped by rounding of u
    assert same_lobe[valid].mean() > 0.9995, same_lobe[valid].mean()
    # per sample within 4x the oracle's own error for >= 99.5 % (GTR1 at small
    # alpha cancels in 1 - a2^(1-u), where either float32 result may land
    # closer by luck), and no worse than the oracle at the 99.9th percentile
    ok = e_gpu <= 4 * e_or + 2e-6
    sel_d = valid & same_lobe
    assert ok[sel_d].mean() > 0.995, ok[sel_d].mean()
    assert np.quantile(e_gpu[sel_d], 0.999) <= 1.25 * np.quantile(e_or[sel_d], 0.999) + 1e-6
    # (b) values at the GPU's direction: weight = f |cos| / pdf (albedo for diffuse)
    f_o, p_o = oracle.bsdf_eval(mats, mi, wi, wog, h)
    f_d, p_d = oracle.bsdf_eval(mats, mi, wi, wog, h, fp64=True)
    sel = valid & (p_o > 0) & (p_d > 0)
    cos_o = np.abs(wog[:, 2:3]).astype(np.float64)
    if kind == pt.PT_MAT_DIFFUSE:
        alb = np.array([list(m.albedo) for m in mats], np.float64)[mi]
        w_o32, w_o64 = alb.astype(np.float32), alb
    else:
        w_o32 = (f_o * cos_o / p_o[:, None]).astype(np.float32)
        w_o64 = f_d.astype(np.float64) * cos_o / p_d[:, None].astype(np.float64)
    sw = parity_stats(wtg[sel], w_o32[sel], w_o64[sel], 1e-6)
    sp = parity_stats(pg[sel], p_o[sel], p_d[sel].astype(np.float64), 1e-6 * float(np.median(np.abs(p_d[sel]))))
    print(kind_name, "weight", sw, "pdf", sp)
    assert_parity(sw)
    assert_parity_ill_conditioned(sp)


@pytest.mark.parametrize("kind_name", ["MIRROR", "DIELECTRIC"])
def test_delta_bsdf_sample_parity(kind_name, pt, scenes, ctx, oracle):
    """Mirror and dielectric scattering: the shading kernels' delta branch
    (shaders/Shaders.hlsl:419-472, one device function for both) queried in
    the local frame from both sides, IOR pairs with extIOR above intIOR as
    well (total internal reflection).  Weight exactly 1 and pdf exactly 0
    (discrete); the Fresnel pick may flip only where u is within rounding of
    Fr; directions no further from FP64 than the float32 oracle's, and
    bit-identical to the float32 oracle's (the same operations in the same
    order, none contracted)."""
    kind = getattr(pt, "PT_MAT_" + kind_name)
    rng = np.random.default_rng(53)
    mats = []
    for _ in range(64):
        m = pt.make_material(kind, (1.0, 1.0, 1.0))
        m.intIOR, m.extIOR = float(rng.uniform(1.0, 2.4)), float(rng.uniform(1.0, 1.8))
        mats.append(m)
    n = N_PAIRS
    wi = scenes.sample_directions(n, 57, upper=False)
    u = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    mi = rng.integers(0, len(mats), n).astype(np.uint32)
    wog, wtg, pg = ctx.bsdf_sample(mats, mi, wi, u, None)
    wo32, wt32, p32 = oracle.bsdf_sample(mats, mi, wi, u, None)
    wo64, _, _ = oracle.bsdf_sample(mats, mi, wi, u, None, fp64=True)
    assert np.all(wtg == 1.0) and np.all(pg == 0.0) and np.all(wt32 == 1.0) and np.all(p32 == 0.0)
    e_gpu = np.abs(wog - wo64).max(1)
    e_or = np.abs(wo32 - wo64).max(1)
    same = e_gpu < 1e-2
    print(kind_name, "same branch", same.mean(), "max err gpu", e_gpu[same].max(), "oracle", e_or[same].max())
    assert same.mean() > 0.9999
    assert (e_gpu <= 4 * e_or + 2e-6)[same].mean() > 0.999
    assert np.quantile(e_gpu[same], 0.999) <= 1.25 * np.quantile(e_or[same], 0.999) + 1e-6
    assert e_gpu[same].max() <= max(2e-5, 2 * e_or[same].max())
    # the device evaluates the delta branch unfused in the oracle's order
    # (reflect, refract, Fresnel, the branch pick): bit for bit the oracle's
    exact = float((wog == wo32).all(1).mean())
    print(kind_name, "directions bit-identical to the float32 oracle:", exact)
    assert np.array_equal(wog, wo32)
    if kind == pt.PT_MAT_DIELECTRIC:
        refracted = np.sign(wog[:, 2]) != np.sign(wi[:, 2])
        assert 0.3 < refracted.mean() < 0.99


def test_phase_sample_parity(ctx, oracle, scenes):
    n = N_PAIRS
    rng = np.random.default_rng(41)
    g = rng.choice(np.array([0.0, 0.3, 0.8, -0.5], np.float32), n)
    wo = scenes.sample_directions(n, 42)
    u = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    wg, pg = ctx.phase_sample(g, wo, u)
    w32, p32 = oracle.phase_sample(g, wo, u)
    w64, p64 = oracle.phase_sample(g, wo, u, fp64=True)
    e_gpu = np.abs(wg - w64).max(1)
    e_or = np.abs(w32 - w64).max(1)
    assert (e_gpu <= 4 * e_or + 2e-6).mean() > 0.999
    assert float(np.quantile(e_gpu, 0.999)) <= 1.25 * float(np.quantile(e_or, 0.999)) + 1e-6
    sp = parity_stats(pg, p32, p64, 1e-6)
    print("phase pdf", sp)
    # the device evaluates the cancelling HG terms unfused, in the oracle's
    # order, so the pdf of the sampled cosine is the oracle's, bit for bit
    assert np.array_equal(pg, p32), sp
    assert_parity(sp)


@pytest.fixture(scope="module")
def sky_scene(scenes):
    return scenes.disney_spheres(64, 48, grid=2, slices=32, rings=17, env_w=512, env_h=256)


def test_envmap_tables_bit_exact(ctx, oracle, sky_scene):
    sc, _ = sky_scene
    ctx.upload(sc)
    oracle.load(sc)
    mg, cg = ctx.env_cdf()
    mo, co = oracle.env_cdf()
    assert np.array_equal(mg, mo) and np.array_equal(cg, co)


@pytest.mark.parametrize("mode", [0, 1])
def test_envmap_sample_pdf_parity(mode, ctx, oracle, sky_scene):
    sc, _ = sky_scene
    ctx.upload(sc)
    oracle.load(sc)
    u = np.random.default_rng(43).uniform(0, 1, (N_PAIRS, 2)).astype(np.float32)
    dg, rg, pg = ctx.env_sample(mode, u)
    do, ro, po = oracle.env_sample(mode, u)
    assert np.abs(dg - do).max() < 1e-5
    assert float(np.quantile(rel_err(pg, po, 1e-6), 0.999)) <= 1e-5
    assert float(np.quantile(rel_err(rg, ro, 1e-6), 0.999)) <= 1e-5
    pg2, rg2 = ctx.env_pdf(mode, do)
    po2, ro2 = oracle.env_pdf(mode, do)
    assert float(np.quantile(rel_err(pg2, po2, 1e-6), 0.999)) <= 1e-5


def test_envmap_guided_search_edges(ctx, oracle, sky_scene):
    """The CDF sampler narrows each binary search with a 256-cell guide table;
    the chosen texel must be the plain search's for every u, including the
    points where the narrowing could go wrong: the cell boundaries k / 256
    (and their float neighbours), and u equal to a CDF entry (the search's
    tie rule), for the marginal and for the conditional rows.  The oracle
    searches the whole CDF."""
    sc, _ = sky_scene
    ctx.upload(sc)
    oracle.load(sc)
    mg, cg = ctx.env_cdf()
    H = mg.size - 1
    cg = cg.reshape(H, -1)
    rng = np.random.default_rng(61)
    k = np.arange(257, dtype=np.float32) / np.float32(256)
    edges = np.concatenate([k, np.nextafter(k, np.float32(0)), np.nextafter(k, np.float32(1))])
    edges = edges[(edges >= 0) & (edges < 1)].astype(np.float32)
    ties_m = mg[(mg >= 0) & (mg < 1)].astype(np.float32)
    # marginal: boundaries and ties, with random column draws
    u1a = np.concatenate([edges, ties_m])
    u2a = rng.uniform(0, 1, u1a.size).astype(np.float32)
    # conditional: random rows, u2 a CDF entry of the row u1 selects, or a boundary
    # (the row as the search picks it: the last entry <= u among all but the last)
    u1b = rng.uniform(0, 1, 20000).astype(np.float32)
    y = np.maximum(np.searchsorted(mg[:-1], u1b, side="right") - 1, 0)
    u2b = cg[y, rng.integers(0, cg.shape[1], y.size)].astype(np.float32)
    u2b = np.where((u2b >= 0) & (u2b < 1), u2b, rng.choice(edges, y.size)).astype(np.float32)
    u2b[::3] = rng.choice(edges, u2b[::3].size)
    u = np.concatenate([np.stack([u1a, u2a], 1), np.stack([u1b, u2b], 1)]).astype(np.float32)
    dg, rg, pg = ctx.env_sample(0, u)
    do, ro, po = oracle.env_sample(0, u)
    assert np.abs(dg - do).max() < 1e-5
    assert float(np.quantile(rel_err(pg, po, 1e-6), 0.999)) <= 1e-5


def test_envmap_wide_rows_plain_search(pt, ctx, oracle, scenes):
    """Rows of 65,536 texels or more do not fit the guide tables' 16-bit
    indices: such an envmap keeps the plain binary search, with the same
    samples as the oracle."""
    env = scenes.sky_envmap(65536, 2, sun_peak=40.0, sun_sigma_deg=4.0)
    m = pt.make_material(pt.PT_MAT_DIFFUSE)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    m.vertexCount, m.indexCount = 3, 3
    sc = pt.Scene(tri, np.array([0, 1, 2]), [m], env_rgb=env)
    ctx.upload(sc)
    oracle.load(sc)
    u = np.random.default_rng(62).uniform(0, 1, (1 << 16, 2)).astype(np.float32)
    dg, rg, pg = ctx.env_sample(0, u)
    do, ro, po = oracle.env_sample(0, u)
    assert np.abs(dg - do).max() < 1e-5
    assert float(np.quantile(rel_err(pg, po, 1e-6), 0.999)) <= 1e-5


@pytest.mark.parametrize("mode", [0, 1])
def test_envmap_sampler_distribution(mode, pt, ctx, scenes):
    """Sampled texels follow lum * sin(theta) (the density both tables encode):
    per-texel counts against expectation, z-scores over texels with >= 200
    expected samples."""
    env = scenes.sky_envmap(64, 32, sun_peak=40.0, sun_sigma_deg=8.0)
    m = pt.make_material(pt.PT_MAT_DIFFUSE)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    m.vertexCount, m.indexCount = 3, 3
    ctx.upload(pt.Scene(tri, np.array([0, 1, 2]), [m], env_rgb=env))
    n = 1 << 22
    u = np.random.default_rng(44 + mode).uniform(0, 1, (n, 2)).astype(np.float32)
    d, _, _ = ctx.env_sample(mode, u)
    phi = np.mod(np.arctan2(d[:, 2], d[:, 0]), 2 * np.pi)
    th = np.arccos(np.clip(d[:, 1], -1, 1))
    H, W = env.shape[:2]
    x = np.minimum((phi / (2 * np.pi) * W).astype(int), W - 1)
    y = np.minimum((th / np.pi * H).astype(int), H - 1)
    cnt = np.bincount(y * W + x, minlength=W * H).astype(np.float64)
    lum = 0.2126 * env[..., 0] + 0.7152 * env[..., 1] + 0.0722 * env[..., 2]
    w = lum * np.sin(np.pi * (np.arange(H) + 0.5) / H)[:, None]
    exp = (w / w.sum()).reshape(-1) * n
    sel = exp >= 200
    z = (cnt[sel] - exp[sel]) / np.sqrt(exp[sel])
    assert np.abs(z).max() < 6.0 and np.mean(z ** 2) < 1.3, (np.abs(z).max(), np.mean(z ** 2))


@pytest.fixture(scope="module")
def bench_scene(scenes):
    """The bench's scene: 64 spheres x 20,480 triangles (1,310,720), treelet-
    restructured 8-wide BVH on the GPU."""
    return scenes.disney_spheres(1280, 720)


@pytest.mark.parametrize("which", ["small", "bench"])
def test_bvh_topology_bit_exact(which, ctx, oracle, scenes, bench_scene):
    if which == "small":
        sc, _ = scenes.disney_spheres(32, 32, grid=3, slices=48, rings=25, env_w=16, env_h=8)
    else:
        sc, _ = bench_scene
    ctx.upload(sc)
    oracle.load(sc)
    mg, og, ng, nwide = ctx.bvh()
    mo, oo, no = oracle.lbvh()
    assert np.array_equal(mg, mo)
    assert np.array_equal(og, oo)
    assert np.array_equal(ng, no)
    assert 0 < nwide < sc.num_triangles


def _surface_rays(sc, rng, n):
    """Rays leaving random points of random triangles (offset 1e-3 along the
    face normal, directions over the sphere): bounce-like rays."""
    P = sc.positions.astype(np.float64)
    f = sc.indices.reshape(-1, 3)
    # indices are per mesh: add each mesh's vertex offset
    off = np.zeros(len(f), np.int64)
    for m in sc.materials:
        off[m.indexOffset // 3:(m.indexOffset + m.indexCount) // 3] = m.vertexOffset
    t = rng.integers(0, len(f), n)
    a, b, c = (P[f[t, k] + off[t]] for k in range(3))
    r1, r2 = rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    s1 = np.sqrt(r1)
    p = a * (1 - s1)[:, None] + b * (s1 * (1 - r2))[:, None] + c * (s1 * r2)[:, None]
    nrm = np.cross(b - a, c - a)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-30
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = p + nrm * np.where((d * nrm).sum(1) > 0, 1e-3, -1e-3)[:, None]
    return o.astype(np.float32), d.astype(np.float32)


@pytest.mark.parametrize("which", ["spheres", "cornell", "hair", "bench", "spheres_plan", "bench_plan"])
def test_trace_parity(which, pt, ctx, oracle, scenes, bench_scene):
    """Closest hits against the oracle's SAH BVH.  The triangle test rounds as
    the oracle's (bit-identical t, u, v), so a ray may disagree only where
    traversal decides: an equal-t tie between triangles, or a hit within
    1e-6 (barycentric) of an edge that one tree's box test grazes.  No other
    disagreement is allowed.  The bench scene's 1,310,720-triangle tree gets
    2^20 rays, half from random points in space, half leaving its surfaces.
    The *_plan cases build the 8-wide tree by the least-area plan, which
    only trees larger than the L2 get by default (PT_DEBUG_WIDE_PLAN)."""
    rng = np.random.default_rng(47)
    n = 200000
    plan = which.endswith("_plan")
    which = which.replace("_plan", "")
    if which == "spheres":
        sc, _ = scenes.disney_spheres(32, 32, grid=3, slices=48, rings=25, env_w=16, env_h=8)
        lo, hi = -6.0, 6.0
    elif which == "cornell":
        sc, _ = scenes.cornell(32, 32)
        lo, hi = -1.0, 2.0
    elif which == "hair":
        sc, _ = scenes.hair_volume(32, 32, strands=400, segments=8, grid_n=16)
        lo, hi = -1.5, 1.5
    else:
        sc, _ = bench_scene
        n = 1 << 20
        lo, hi = sc.positions.min(0) - 1.0, sc.positions.max(0) + 1.0
    ctx.debug_set(pt.PT_DEBUG_WIDE_PLAN, 1 if plan else 0)
    try:
        ctx.upload(sc)
    finally:
        ctx.debug_set(pt.PT_DEBUG_WIDE_PLAN, 0)
    oracle.load(sc)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = scenes.sample_directions(n, 48)
    if which == "bench":
        o[n // 2:], d[n // 2:] = _surface_rays(sc, rng, n - n // 2)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7], rays[:, 7] = o, 0.0, d, 1e20
    hg = ctx.trace_closest(rays)
    ho = oracle.trace_closest(rays)
    same_hit = hg["hit"] == ho["hit"]
    both = (hg["hit"] == 1) & (ho["hit"] == 1)
    same_prim = (hg["mesh"] == ho["mesh"]) & (hg["prim"] == ho["prim"])

    def near_edge(h):
        return (h["hit"] == 1) & (np.minimum(np.minimum(h["u"], h["v"]), 1 - h["u"] - h["v"]) < 1e-6)

    tie = both & (hg["t"] == ho["t"])
    exempt = near_edge(hg) | near_edge(ho) | tie
    bad = ~(same_hit & (~both | same_prim))
    print(which, "rays", n, "hits", int(both.sum()), "disagreements", int(bad.sum()), "ties", int((bad & tie).sum()),
          "within 1e-6 of an edge", int((bad & ~tie & exempt).sum()), "unexplained", int((bad & ~exempt).sum()))
    assert (bad & ~exempt).sum() == 0, int((bad & ~exempt).sum())
    assert bad.mean() < 1e-4
    # the same triangle at the same distance, bit for bit
    tt = both & same_prim
    assert np.array_equal(hg["t"][tt], ho["t"][tt])
    assert np.array_equal(hg["u"][tt], ho["u"][tt]) and np.array_equal(hg["v"][tt], ho["v"][tt])
    # shadow rays: occlusion within half the closest-hit distance
    rays[:, 7] = np.where(ho["hit"] == 1, ho["t"] * 0.5, 10.0)
    og, _ = ctx.trace_shadow(rays)
    oo, _ = oracle.trace_shadow(rays)
    print(which, "shadow disagreements", int((og != oo).sum()))
    assert (og != oo).mean() < 1e-4
