"""Resampled importance sampling of area lights (PT_RENDER_RIS_NEE; the
reference's USE_RIS=1 build, shaders/Emitter.hlsli:155-271): eight emitter
candidates through a one-sample reservoir, the survivor shadow-tested and
MIS-weighted with its solid-angle pdf.

CPU: the oracle restatement equals the reference's RIS build bit for bit
(tests/test_oracle_ref.py::test_ris_render_identical).  GPU: per-path and
image parity with the oracle on a scene of four uneven lights; RIS and the
default MIS estimator converge to the same image; RIS in a batch."""

import numpy as np
import pytest


def mean_img(s):
    return s[..., :3] / np.maximum(s[..., 3:4], 1.0)


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


@pytest.mark.gpu
def test_ris_render_parity(pt, scenes, ctx, oracle):
    sc, cam = scenes.cornell(64, 64, many_lights=True)
    ctx.upload(sc)
    oracle.load(sc)
    P = pt.render_params(64, 64, 1, cam, max_depth=8, flags=pt.PT_RENDER_RIS_NEE)
    g, _, _ = ctx.render(P)
    _, per, _ = oracle.render(P, per_path=True)
    close = np.abs(g[..., :3] - per[0]) <= 1e-3 * np.maximum(np.abs(per[0]), 1e-2)
    assert close.all(-1).mean() > 0.97, close.all(-1).mean()
    P16 = pt.render_params(64, 64, 16, cam, max_depth=8, flags=pt.PT_RENDER_RIS_NEE)
    g16, _, _ = ctx.render(P16)
    o16, _, _ = oracle.render(P16)
    assert relmse(mean_img(g16), mean_img(o16)) < 1e-3


@pytest.mark.gpu
def test_ris_and_mis_agree(pt, scenes, ctx):
    """Both estimators are unbiased: their 4096-spp images agree in the mean
    and block by block (8 x 8 pixel blocks average out the small, bright
    lights' remaining noise)."""
    sc, cam = scenes.cornell(64, 64, many_lights=True)
    ctx.upload(sc)
    a, _, _ = ctx.render(pt.render_params(64, 64, 4096, cam, max_depth=8, flags=pt.PT_RENDER_RIS_NEE))
    b, _, _ = ctx.render(pt.render_params(64, 64, 4096, cam, max_depth=8, sample_offset=1 << 16))
    ma, mb = mean_img(a), mean_img(b)
    assert abs(float(ma.mean()) / float(mb.mean()) - 1.0) < 1e-2
    ba = ma.reshape(8, 8, 8, 8, 3).mean((1, 3))
    bb = mb.reshape(8, 8, 8, 8, 3).mean((1, 3))
    assert relmse(ba, bb) < 2e-3, relmse(ba, bb)


@pytest.mark.gpu
def test_ris_in_batch(pt, scenes, ctx):
    sc, cam = scenes.cornell(64, 64, many_lights=True)
    ctx.upload(sc)
    reqs = [pt.render_params(64, 64, 2, cam, max_depth=8, flags=pt.PT_RENDER_RIS_NEE),
            pt.render_params(40, 24, 3, cam, max_depth=6, sample_offset=9, flags=pt.PT_RENDER_RIS_NEE)]
    films, _, _ = ctx.render_batch(reqs)
    for P, (s, c) in zip(reqs, films):
        s1, c1, _ = ctx.render(pt.render_params(P.width, P.height, P.spp, P.camera, max_depth=P.max_depth,
                                                sample_offset=P.sample_offset, flags=pt.PT_RENDER_RIS_NEE))
        assert np.array_equal(s, s1) and np.array_equal(c, c1)
