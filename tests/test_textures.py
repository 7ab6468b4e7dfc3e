"""Material textures and alpha cut-outs (shaders/Shaders.hlsl:232-315,
shaders/RayQueryTrace.hlsli:50-62,100-112).

CPU: invariants of the oracle's restatement — a white sRGB albedo map equals
an untextured albedo of 1, an alpha map of 0 removes its mesh, an alpha map
of 1 leaves it opaque, and textures change the image.
GPU: libpt against the oracle on a scene with every map (per path and by
relMSE), the same invariants on the device, and the alpha test in the batch
trace entry point.  Texture filtering is trilinear float arithmetic on both
sides (the reference's hardware filtering is unpinned), so per-path parity
has the tolerance of the other render tests, not bit equality.
"""

import copy

import numpy as np
import pytest


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def mean_img(s):
    return s[..., :3] / np.maximum(s[..., 3:4], 1.0)


def rebuilt(pt, sc, mats=None, textures=None, drop=None):
    """The scene's arrays with changed materials / textures, or without mesh `drop`."""
    mats = [copy.copy(m) for m in (sc.materials if mats is None else mats)]
    pos, idx = sc.positions, sc.indices
    nrm, uv, tan = sc.normals, sc.texcoords, sc.tangents
    if drop is not None:
        m = mats[drop]
        keep_i = np.ones(len(idx), bool)
        keep_i[m.indexOffset:m.indexOffset + m.indexCount] = False
        idx = idx[keep_i]
        for k in mats[drop + 1:]:
            k.indexOffset -= m.indexCount
        mats = mats[:drop] + mats[drop + 1:]
    tex = list(zip(sc.tex_arrays, sc.tex_srgb)) if textures is None else textures
    return pt.Scene(pos, idx, mats, normals=nrm, texcoords=uv, tangents=tan, env_rgb=sc.env_rgb,
                    env_scale=sc.env_scale, textures=tex)


def maps_with_flags(scenes):
    return scenes.texture_maps(0)


# ---------------------------------------------------------------------------- CPU (oracle)
def test_oracle_white_albedo_map_equals_untextured(pt, scenes, oracle):
    sc, cam = scenes.textured_scene(48, 36)
    maps = maps_with_flags(scenes)
    mats = list(sc.materials)
    for m in mats:
        m.albedoTexIndex = m.normalTexIndex = m.roughnessTexIndex = m.specularTexIndex = pt.PT_NO_TEXTURE
        m.alphaTexIndex = pt.PT_NO_TEXTURE
    plain = rebuilt(pt, sc, mats=mats, textures=maps)
    mats_w = [copy.copy(m) for m in mats]
    mats_w[1].albedo[:] = (1.0, 1.0, 1.0)
    white = np.full((4, 4, 4), 255, np.uint8)
    tex_w = maps + [(white, True)]
    mats_t = [copy.copy(m) for m in mats_w]
    mats_t[1].albedoTexIndex = len(maps)
    P = pt.render_params(48, 36, 2, cam, max_depth=6)
    oracle.load(rebuilt(pt, sc, mats=mats_w, textures=maps))
    a, _, _ = oracle.render(P)
    oracle.load(rebuilt(pt, sc, mats=mats_t, textures=tex_w))
    b, _, _ = oracle.render(P)
    assert np.array_equal(a, b)
    oracle.load(plain)
    c, _, _ = oracle.render(P)
    assert not np.array_equal(a, c)  # the floor albedo changed 0.7 -> 1


@pytest.mark.parametrize("alpha", [0, 255])
def test_oracle_alpha_extremes(alpha, pt, scenes, oracle):
    """Alpha 0 everywhere: the cut-out quad vanishes (equals the scene without
    it); alpha 1 everywhere: it is opaque (equals no alpha map)."""
    sc, cam = scenes.textured_scene(48, 36)
    maps = maps_with_flags(scenes)
    const = np.full((8, 8, 4), alpha, np.uint8)
    tex = maps[:5] + [const]
    P = pt.render_params(48, 36, 2, cam, max_depth=6)
    oracle.load(rebuilt(pt, sc, textures=tex))
    a, _, _ = oracle.render(P)
    if alpha == 0:
        oracle.load(rebuilt(pt, sc, textures=tex, drop=2))
    else:
        mats = [copy.copy(m) for m in sc.materials]
        mats[2].alphaTexIndex = pt.PT_NO_TEXTURE
        oracle.load(rebuilt(pt, sc, mats=mats, textures=tex))
    b, _, _ = oracle.render(P)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()


def test_oracle_textures_change_the_image(pt, scenes, oracle):
    sc, cam = scenes.textured_scene(48, 36)
    P = pt.render_params(48, 36, 4, cam, max_depth=6)
    oracle.load(sc)
    a, _, _ = oracle.render(P)
    mats = [copy.copy(m) for m in sc.materials]
    mats[0].normalTexIndex = pt.PT_NO_TEXTURE
    oracle.load(rebuilt(pt, sc, mats=mats, textures=maps_with_flags(scenes)))
    b, _, _ = oracle.render(P)
    assert relmse(mean_img(a), mean_img(b)) > 1e-4  # the normal map matters
    assert np.isfinite(a).all()


# ---------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_textured_render_parity(pt, scenes, ctx, oracle):
    sc, cam = scenes.textured_scene(96, 72)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(96, 72, 1, cam, max_depth=8)
    g, _, _ = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    close = np.abs(g[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)
    assert close.all(-1).mean() > 0.97, close.all(-1).mean()
    P16 = pt.render_params(96, 72, 16, cam, max_depth=8)
    g16, _, _ = ctx.render(P16)
    o16, _, _ = oracle.render(P16)
    assert relmse(mean_img(g16), mean_img(o16)) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("alpha", [0, 255])
def test_alpha_extremes_gpu(alpha, pt, scenes, ctx):
    sc, cam = scenes.textured_scene(64, 48)
    maps = maps_with_flags(scenes)
    tex = maps[:5] + [np.full((8, 8, 4), alpha, np.uint8)]
    P = pt.render_params(64, 48, 2, cam, max_depth=6)
    ctx.upload(rebuilt(pt, sc, textures=tex))
    a, _, _ = ctx.render(P)
    if alpha == 0:
        ctx.upload(rebuilt(pt, sc, textures=tex, drop=2))
    else:
        mats = [copy.copy(m) for m in sc.materials]
        mats[2].alphaTexIndex = pt.PT_NO_TEXTURE
        ctx.upload(rebuilt(pt, sc, mats=mats, textures=tex))
    b, _, _ = ctx.render(P)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()


@pytest.mark.gpu
def test_alpha_trace_parity(pt, scenes, ctx, oracle):
    """Batch closest-hit / shadow traces through the alpha-cut quad: the same
    hits and occlusions as the oracle (seed = ray index on both sides)."""
    sc, _ = scenes.textured_scene()
    ctx.upload(sc)
    oracle.load(sc)
    rng = np.random.default_rng(4)
    n = 20000
    o = np.stack([rng.uniform(-0.7, 0.7, n), rng.uniform(-0.7, 0.7, n), np.full(n, 3.0)], 1)
    d = np.tile([0.0, 0.0, -1.0], (n, 1))
    rays = np.concatenate([o, np.full((n, 1), 0.0), d, np.full((n, 1), 1.9)], 1).astype(np.float32)
    hg, ho = ctx.trace_closest(rays), oracle.trace_closest(rays)
    assert 0.2 < hg["hit"].mean() < 0.9  # the cut-out lets part of the rays through
    same = (hg["hit"] == ho["hit"]) & ((hg["hit"] == 0) | ((hg["mesh"] == ho["mesh"]) & (hg["prim"] == ho["prim"])))
    assert same.mean() > 0.999
    occ_g, _ = ctx.trace_shadow(rays)
    occ_o, _ = oracle.trace_shadow(rays)
    assert (np.asarray(occ_g) == np.asarray(occ_o)).mean() > 0.999
