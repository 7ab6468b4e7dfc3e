"""The device error paths, exercised without faulting the GPU.

Kernels never trap: bounded checks raise bits in a device flag that the host
turns into PT_E_DEVICE, and the context stays usable.  pt_debug_set (a test
hook) makes two of those checks fire on purpose:

* a shadow-ray queue smaller than the NEE rays of a render: appends beyond
  it are dropped and flagged (queue overflow), and the shadow kernel reads
  only what was stored;
* the radiance-cache kernels' bounded mbarrier wait: with the stall hook
  every CTA first waits a few polls on a barrier nothing arrives at, before
  it issues any copy or tensor-core work, gives up, frees its TMEM and
  returns.  Had TMEM not been freed, the next cache kernel could not
  allocate it; the next calls must run and give the clean results.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_hook_arguments_checked(pt, ctx):
    with pytest.raises(pt.PTError):
        ctx.debug_set(99, 1)
    with pytest.raises(pt.PTError):
        ctx.debug_set(pt.PT_DEBUG_SHADOW_QUEUE_CAP, 1 << 40)


def test_shadow_queue_overflow_reported_then_recovers(pt, scenes):
    sc, cam = scenes.cornell(64, 64)
    ctx = pt.Context(0)
    try:
        ctx.upload(sc)
        P = pt.render_params(64, 64, 4, cam, max_depth=8)
        clean, _, st = ctx.render(P)
        assert st.shadow_rays > 4000  # the cap below is far under what the render queues
        ctx.debug_set(pt.PT_DEBUG_SHADOW_QUEUE_CAP, 1000)
        with pytest.raises(pt.PTError) as e:
            ctx.render(P)
        assert "-5" in str(e.value) and "queue overflow" in str(e.value)
        ctx.debug_set(pt.PT_DEBUG_SHADOW_QUEUE_CAP, 0)
        again, _, _ = ctx.render(P)
        assert np.array_equal(again, clean)
    finally:
        ctx.close()


def test_cache_wait_timeout_reported_then_recovers(pt):
    ctx = pt.Context(0)
    try:
        ctx.cache_init(pt.cache_params(seed=3, bbox=((0, 0, 0), (1, 1, 1))))
        rng = np.random.default_rng(9)
        n = 50000  # several tiles per SM for the inference grid
        f = rng.uniform(-1, 1, (n, pt.PT_CACHE_FEATURES)).astype(np.float32)
        f[:, 49], f[:, 50:] = 1.0, 0.0
        t = rng.uniform(0, 2, (n, 3)).astype(np.float32)
        y0 = ctx.cache_infer(f)
        g0, l0 = ctx.cache_gradient(f, t)
        ctx.debug_set(pt.PT_DEBUG_CACHE_STALL, 64)
        for call in (lambda: ctx.cache_infer(f), lambda: ctx.cache_gradient(f, t)):
            with pytest.raises(pt.PTError) as e:
                call()
            assert "-5" in str(e.value) and "wait timed out" in str(e.value)
        ctx.debug_set(pt.PT_DEBUG_CACHE_STALL, 0)
        y1 = ctx.cache_infer(f)
        g1, l1 = ctx.cache_gradient(f, t)
        assert np.array_equal(y0, y1)
        # gradient sums use float atomics: the same up to summation order (a
        # few near-cancelling components move by more than their own size)
        assert np.linalg.norm(g1 - g0) <= 1e-5 * np.linalg.norm(g0) and abs(l0 - l1) <= 1e-4 * abs(l0)
    finally:
        ctx.close()
