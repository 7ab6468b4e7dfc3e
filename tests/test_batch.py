"""Batched requests (pt_render_batch, pt_batch_autotune): many requests of
one scene with their own image size, spp, sample offset, depth and camera
rendered as one wavefront.  Each request's film must equal the same request
rendered alone by pt_render, bit for bit: the batch assigns every path the
same pixel, sample index and random numbers, and each film adds its pixel's
samples in sample order.  No counterpart in the reference (one dispatch per
frame); the single-request renders are themselves checked against the
oracle by the render tests."""

import ctypes as C

import numpy as np
import pytest


def look(scenes, eye, target, aspect):
    return scenes.look_at_camera(eye, target, (0, 1, 0), 40.0, aspect)


def cornell_requests(pt, scenes, wave=0):
    """Uneven requests: sizes 16x16 .. 96x64, 1..24 spp, depths 5..8."""
    spec = [(96, 64, 3, 8, 0), (32, 32, 24, 8, 100), (50, 30, 2, 5, 7), (16, 16, 16, 8, 3), (80, 40, 1, 6, 0),
            (64, 64, 4, 8, 40), (20, 36, 9, 7, 11)]
    out = []
    for k, (w, h, spp, depth, off) in enumerate(spec):
        cam = look(scenes, (0.1 * k - 0.3, 0.5 + 0.05 * k, 2.2 + 0.1 * k), (0, 0.45, 0), w / h)
        out.append(pt.render_params(w, h, spp, cam, max_depth=depth, sample_offset=off, wave_paths=wave))
    return out


def render_alone(pt, ctx, P):
    Q = pt.render_params(P.width, P.height, P.spp, P.camera, max_depth=P.max_depth, sample_offset=P.sample_offset,
                         rng_kind=P.rng_kind, env_sampling=P.env_sampling)
    s, c, _ = ctx.render(Q)
    return s, c


def assert_batch_equals_single(pt, ctx, reqs, films):
    for P, (s, c) in zip(reqs, films):
        s1, c1 = render_alone(pt, ctx, P)
        assert np.array_equal(s, s1), (P.width, P.height, P.spp, np.abs(s - s1).max())
        assert np.array_equal(c, c1)


# ---------------------------------------------------------------------------- CPU
def test_batch_abi_sizes(pt):
    assert pt.pt_request.film.offset % 8 == 0
    assert C.sizeof(pt.pt_batch_tuning) == 16 + 16 * 12


# ---------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("wave", [0, 4096, 20000])
def test_batch_equals_single_renders(pt, scenes, ctx, wave):
    """One wave, and waves of 4096 / 20000 paths that split requests and
    hold pieces of several."""
    sc, _ = scenes.cornell(64, 64)
    ctx.upload(sc)
    reqs = cornell_requests(pt, scenes, wave)
    films, ms, st = ctx.render_batch(reqs)
    assert st.paths == sum(P.width * P.height * P.spp for P in reqs)
    assert all(np.all(f[0][..., 3] == P.spp) for P, f in zip(reqs, films))
    assert_batch_equals_single(pt, ctx, reqs, films)
    if wave:
        # requests finish in path order (shortest first): completion times follow
        order = np.argsort([P.width * P.height * P.spp for P in reqs], kind="stable")
        assert np.all(ms > 0) and np.all(np.diff(ms[order]) >= -1e-3)
        assert ms[order[0]] < ms[order[-1]]
        assert st.waves == -(-st.paths // wave)


@pytest.mark.gpu
def test_batch_device_films_and_accumulation(pt, scenes, ctx):
    """Device films, and a second batch adding more samples into them equals
    a single render of all the samples."""
    import torch

    sc, _ = scenes.cornell(64, 64)
    ctx.upload(sc)
    reqs = cornell_requests(pt, scenes)
    films = [(torch.zeros((P.height, P.width, 4), device="cuda"), torch.zeros((P.height, P.width, 4), device="cuda"))
             for P in reqs]
    ptrs = [(a.data_ptr(), b.data_ptr()) for a, b in films]
    ctx.render_batch(reqs, ptrs, pt.PT_MEM_DEVICE)
    more = []
    for P in reqs:
        Q = pt.render_params(P.width, P.height, P.spp + 1, P.camera, max_depth=P.max_depth,
                             sample_offset=P.sample_offset + P.spp)
        more.append(Q)
    ctx.render_batch(more, ptrs, pt.PT_MEM_DEVICE)
    for P, (a, b) in zip(reqs, films):
        Q = pt.render_params(P.width, P.height, P.spp, P.camera, max_depth=P.max_depth, sample_offset=P.sample_offset)
        s, c, _ = ctx.render(Q)
        Q2 = pt.render_params(P.width, P.height, P.spp + 1, P.camera, max_depth=P.max_depth,
                              sample_offset=P.sample_offset + P.spp)
        s, c, _ = ctx.render(Q2, s, c)
        assert np.array_equal(a.cpu().numpy(), s) and np.array_equal(b.cpu().numpy(), c)


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["textured", "disney", "volume"])
def test_batch_other_scenes(pt, scenes, ctx, scene):
    """Texture LOD uses each request's own image size; media scenes run the
    inline-shadow shading kernel; both per request as alone."""
    if scene == "textured":
        sc, cam = scenes.textured_scene(64, 48)
    elif scene == "disney":
        sc, cam = scenes.disney_spheres(96, 64, grid=3, slices=32, rings=17, env_w=256, env_h=128)
    else:
        sc, cam = scenes.hair_volume(48, 48, strands=200, segments=8, grid_n=32)
    ctx.upload(sc)
    reqs = [pt.render_params(64, 48, 2, cam, max_depth=8), pt.render_params(24, 40, 5, cam, max_depth=6,
                                                                            sample_offset=9),
            pt.render_params(128, 96, 1, cam, max_depth=8, sample_offset=3, wave_paths=5000)]
    for P in reqs:
        P.wave_paths = 5000
    films, _, _ = ctx.render_batch(reqs)
    assert_batch_equals_single(pt, ctx, reqs, films)


@pytest.mark.gpu
def test_batch_autotune(pt, scenes, ctx):
    sc, _ = scenes.cornell(64, 64)
    ctx.upload(sc)
    reqs = cornell_requests(pt, scenes)
    films = [(np.full((P.height, P.width, 4), 7.0, np.float32), np.zeros((P.height, P.width, 4), np.float32))
             for P in reqs]
    t = ctx.batch_autotune(reqs, films)
    assert t.candidates >= 2 and t.ms > 0 and t.wave_paths > 0
    assert t.ms == min(t.candidate_ms[:t.candidates])
    assert all(np.all(f[0] == 7.0) for f in films)  # the tuner leaves the films alone
    out, _, _ = ctx.render_batch(reqs)
    assert_batch_equals_single(pt, ctx, reqs, out)


@pytest.mark.gpu
def test_batch_invalid_requests(pt, scenes, ctx):
    sc, cam = scenes.cornell(64, 64)
    ctx.upload(sc)
    a = pt.render_params(32, 32, 2, cam, max_depth=4)
    b = pt.render_params(32, 32, 2, cam, max_depth=4, rng_kind=pt.PT_RNG_PCG_HASH)
    with pytest.raises(pt.PTError, match="agree"):
        ctx.render_batch([a, b])
    big = pt.render_params(4096, 4096, 1, cam, max_depth=4)
    with pytest.raises(pt.PTError, match="PT_BATCH_MAX_PIXELS"):
        ctx.render_batch([big], [(np.zeros(1, np.float32), np.zeros(1, np.float32))])
    reqs = (pt.pt_request * 1)()
    assert ctx.L.pt_render_batch(ctx.h, reqs, 0, None, None) == -1
