"""pt_bsdf_eval_batch_noalloc (static device staging, no allocation, no
context) against pt_bsdf_eval_batch on the same inputs.  Both run the same
evaluation kernel, so results must agree to 1e-6 relative; the calls come in a
row with different sizes and optional inputs, so stale staging contents from
an earlier call would show."""

import ctypes as C

import numpy as np
import pytest

PT_E_INVALID, PT_E_LIMIT = -1, -7
MAX_Q, MAX_M = 65536, 256


def _noalloc(pt):
    L = pt.lib()
    F = C.POINTER(C.c_float)
    U = C.POINTER(C.c_uint32)
    fn = L.pt_bsdf_eval_batch_noalloc
    fn.argtypes = [C.c_void_p, C.POINTER(pt.pt_material), C.c_uint32, U, F, F, F, C.c_size_t, F, F, C.c_uint32]
    fn.restype = C.c_int
    return fn


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _up(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_uint32))


def _call(pt, mats, mi, wi, wo, h, n=None):
    n = len(wi) if n is None else n
    ma = (pt.pt_material * len(mats))(*mats)
    f = np.full((len(wi), 3), np.nan, np.float32)
    pdf = np.full(len(wi), np.nan, np.float32)
    rc = _noalloc(pt)(None, ma, len(mats), _up(mi), _fp(wi), _fp(wo), _fp(h), n, _fp(f), _fp(pdf), 0)
    return rc, f, pdf


def _materials(pt, rng):
    mats = []
    for k in range(12):
        kind = [pt.PT_MAT_DIFFUSE, pt.PT_MAT_MICROFACET, pt.PT_MAT_DISNEY, pt.PT_MAT_HAIR][k % 4]
        m = pt.make_material(kind, tuple(rng.uniform(0.05, 1.0, 3)))
        if kind == pt.PT_MAT_DISNEY:
            m.roughness, m.metallic, m.clearcoat, m.sheen = rng.uniform(0.05, 1.0, 4)
        elif kind == pt.PT_MAT_MICROFACET:
            m.alpha = rng.uniform(0.05, 0.8)
        elif kind == pt.PT_MAT_HAIR:
            m.roughness, m.betaN, m.alpha, m.intIOR = 0.3, 0.3, 2.0, 1.55
        mats.append(m)
    return mats


def test_limits_rejected_before_any_device_work(pt):
    """Sizes above the static array's capacity and bad arguments come back as
    status codes (checked on the host; no device needed)."""
    m = [pt.make_material(pt.PT_MAT_DIFFUSE, (0.5, 0.5, 0.5))]
    wi = np.zeros((MAX_Q + 1, 3), np.float32)
    rc, _, _ = _call(pt, m, None, wi, wi, None)
    assert rc == PT_E_LIMIT
    rc, _, _ = _call(pt, m * (MAX_M + 1), None, wi[:4], wi[:4], None)
    assert rc == PT_E_LIMIT
    f = np.zeros((4, 3), np.float32)
    assert _noalloc(pt)(None, None, 1, None, _fp(wi), _fp(wi), None, 4, _fp(f), _fp(f), 0) == PT_E_INVALID


@pytest.mark.gpu
def test_noalloc_matches_staged_entry_point(pt, scenes, ctx):
    rng = np.random.default_rng(5)
    mats = _materials(pt, rng)
    # call 1: the largest batch, every optional input present
    n1 = MAX_Q
    wi = scenes.sample_directions(n1, 31, upper=False)
    wo = scenes.sample_directions(n1, 32, upper=False)
    mi = rng.integers(0, len(mats), n1).astype(np.uint32)
    h = rng.uniform(-0.9, 0.9, n1).astype(np.float32)
    rc, f1, p1 = _call(pt, mats, mi, wi, wo, h)
    assert rc == 0
    g1, q1 = ctx.bsdf_eval(mats, mi, wi, wo, h)
    assert np.allclose(f1, g1, rtol=1e-6, atol=0) and np.allclose(p1, q1, rtol=1e-6, atol=0)
    # call 2, right after: fewer queries, one material, no mat_index and no h
    # (the kernel must not pick up call 1's staged mat_index or h)
    n2 = 1000
    hair = [mats[3]]
    wi2 = scenes.sample_directions(n2, 33, upper=False)
    wo2 = scenes.sample_directions(n2, 34, upper=False)
    rc, f2, p2 = _call(pt, hair, None, wi2, wo2, None)
    assert rc == 0
    g2, q2 = ctx.bsdf_eval(hair, None, wi2, wo2, None)
    assert np.allclose(f2, g2, rtol=1e-6, atol=0) and np.allclose(p2, q2, rtol=1e-6, atol=0)
    assert np.isfinite(f2).all() and np.isfinite(p2).all()
    # the property the entry point exists for: once warm, calls of any size up
    # to the limit leave the device's free memory exactly where it was
    import torch

    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for n in (17, 4096, MAX_Q, 1):
        rc, f3, _ = _call(pt, mats, mi[:n], wi[:n], wo[:n], h[:n])
        assert rc == 0 and np.allclose(f3, g1[:n], rtol=1e-6, atol=0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.gpu
def test_noalloc_device_arrays_in_place(pt, scenes, ctx):
    import torch

    rng = np.random.default_rng(6)
    mats = _materials(pt, rng)
    n = 4096
    wi = scenes.sample_directions(n, 41)
    wo = scenes.sample_directions(n, 42)
    mi = rng.integers(0, len(mats), n).astype(np.uint32)
    g, q = ctx.bsdf_eval(mats, mi, wi, wo, None)
    ma = (pt.pt_material * len(mats))(*mats)
    dm = torch.frombuffer(bytearray(bytes(ma)), dtype=torch.uint8).cuda()
    dmi = torch.from_numpy(mi.view(np.int32)).cuda()
    dwi, dwo = torch.from_numpy(wi).cuda(), torch.from_numpy(wo).cuda()
    df = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    dp = torch.empty(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    fn = _noalloc(pt)
    fn.argtypes = [C.c_void_p] * 2 + [C.c_uint32] + [C.c_void_p] * 4 + [C.c_size_t] + [C.c_void_p] * 2 + [C.c_uint32]
    rc = fn(None, dm.data_ptr(), len(mats), dmi.data_ptr(), dwi.data_ptr(), dwo.data_ptr(), None, n,
            df.data_ptr(), dp.data_ptr(), 1)
    assert rc == 0
    assert np.allclose(df.cpu().numpy(), g, rtol=1e-6, atol=0) and np.allclose(dp.cpu().numpy(), q, rtol=1e-6, atol=0)
