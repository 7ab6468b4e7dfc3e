"""Subsurface material (type 6; shaders/Shaders.hlsl:515-611,
shaders/Subsurface.hlsli:24-144, shaders/Material.hlsli:48-58,92-100): a
rough dielectric entry sampled through a Beckmann half vector with a Fresnel
choice, NEE with the entry lobe, and a random walk through the interior
medium (free flights, HG scattering, Fresnel at the boundary, Russian
roulette) that leaves the mesh elsewhere.

CPU: the oracle restatement gives the reference shader build's image bit for
bit (tests/test_oracle_ref.py::test_render_identical[subsurface]); here, the
walk changes the image and energy stays bounded.  GPU: per-path and image
parity with the oracle, the subsurface scene in a batch, and the entry lobe's
eval / pdf (tests/test_gpu_parity.py::test_bsdf_eval_parity[SUBSURFACE])."""

import numpy as np
import pytest


def mean_img(s):
    return s[..., :3] / np.maximum(s[..., 3:4], 1.0)


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def test_oracle_walk_changes_the_sphere(pt, scenes, oracle):
    sc, cam = scenes.subsurface_scene(48, 40)
    P = pt.render_params(48, 40, 8, cam, max_depth=8)
    oracle.load(sc)
    a, _, _ = oracle.render(P)
    plain, _ = scenes.cornell(48, 40)
    oracle.load(plain)
    b, _, _ = oracle.render(P)
    ma, mb = mean_img(a), mean_img(b)
    assert np.isfinite(ma).all()
    assert (np.abs(ma - mb).max(-1) > 1e-3).mean() > 0.1
    assert ma.max() < 50.0


@pytest.mark.gpu
@pytest.mark.parametrize("mfp,g", [(0.08, 0.2), (0.5, -0.3), (0.02, 0.0)])
def test_subsurface_render_parity(pt, scenes, ctx, oracle, mfp, g):
    sc, cam = scenes.subsurface_scene(64, 64, mfp=mfp, g=g)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(64, 64, 1, cam, max_depth=8)
    gi, _, _ = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    close = np.abs(gi[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)
    assert close.all(-1).mean() > 0.97, close.all(-1).mean()
    P16 = pt.render_params(64, 64, 16, cam, max_depth=8)
    g16, _, _ = ctx.render(P16)
    o16, _, _ = oracle.render(P16)
    assert relmse(mean_img(g16), mean_img(o16)) < 1e-3


@pytest.mark.gpu
def test_subsurface_in_batch(pt, scenes, ctx):
    sc, cam = scenes.subsurface_scene(64, 64)
    ctx.upload(sc)
    reqs = [pt.render_params(64, 64, 2, cam, max_depth=8), pt.render_params(32, 48, 3, cam, max_depth=6,
                                                                            sample_offset=5)]
    films, _, _ = ctx.render_batch(reqs)
    for P, (s, c) in zip(reqs, films):
        s1, c1, _ = ctx.render(pt.render_params(P.width, P.height, P.spp, P.camera, max_depth=P.max_depth,
                                                sample_offset=P.sample_offset))
        assert np.array_equal(s, s1) and np.array_equal(c, c1)
