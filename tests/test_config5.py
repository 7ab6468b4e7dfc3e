"""The radiance-cache scene (configuration 5): displaced icosphere instances
with Disney and hair materials, ground and wall, a fog box and the sky
envmap.  CPU: generator invariants.  GPU, on a small version of the scene
(the same materials, medium and envmap; 4 instances of subdivision 2): plain
and constant-cache renders against the oracle (the medium routes the scene
through the inline-trace shading kernel)."""

import numpy as np
import pytest

from oracle import radiance_cache as rc


def mean_img(s):
    return s[..., :3] / np.maximum(s[..., 3:4], 1.0)


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def test_generator(pt, scenes):
    sc, cam = scenes.radiance_cache_scene(64, 36, instances=9, subdiv=3)
    assert sc.num_triangles == 9 * 20 * 4 ** 3 + 4
    n = sc.normals.reshape(-1, 3)[: 9 * (10 * 4 ** 3 + 2)]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-5)
    types = [m.type for m in sc.materials]
    assert types.count(pt.PT_MAT_HAIR) == 1 and types.count(pt.PT_MAT_DISNEY) == 9
    big_side = int(np.ceil(np.sqrt(122)))
    assert 122 * 20 * 4 ** 6 + 4 == 9994244 and big_side == 12


@pytest.fixture(scope="module")
def small(scenes):
    return scenes.radiance_cache_scene(64, 36, instances=4, subdiv=2)


@pytest.mark.gpu
def test_plain_render_parity(pt, ctx, oracle, small):
    sc, cam = small
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(64, 36, 1, cam, max_depth=16)
    g, _, _ = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    close = np.abs(g[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)
    assert close.all(-1).mean() > 0.95, close.all(-1).mean()
    P16 = pt.render_params(64, 36, 64, cam, max_depth=16)
    g16, _, _ = ctx.render(P16)
    o16, _, _ = oracle.render(P16)
    assert relmse(mean_img(g16), mean_img(o16)) < 2e-3


@pytest.mark.gpu
def test_constant_cache_render_parity(pt, ctx, oracle, small):
    sc, cam = small
    ctx.upload(sc)
    oracle.load(sc)
    value = np.float32([0.25, 0.5, 0.125])
    ctx.cache_init(pt.cache_params(flags=pt.PT_CACHE_NO_TRAIN, rough_threshold=0.3))
    try:
        ctx.cache_weights(rc.constant_weights(value))
        P = pt.render_params(64, 36, 2, cam, max_depth=16, flags=pt.PT_RENDER_RADIANCE_CACHE)
        g, _, _ = ctx.render(P)
        o, _ = oracle.render_cached(P, value, 0.3)
        close = np.abs(mean_img(g) - mean_img(o)) <= 1e-3 * np.maximum(np.abs(mean_img(o)), 1e-2)
        assert close.all(-1).mean() > 0.95, close.all(-1).mean()
    finally:
        ctx.cache_release()
