"""ctypes binding of the CPU oracle (liboracle.so) and of the reference's shader
code built for the CPU (oracle/_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker; the product never calls it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")
REF_RIS_SO = os.path.join(HERE, "_ref", "libref_ris.so")  # the reference's USE_RIS=1 build
# the reference checkout (read only where it is present): $PBRT_REFERENCE_ROOT,
# default /root/reference
REF_ROOT = os.environ.get("PBRT_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "shaders")


def build_oracle(quiet=True) -> str:
    """Compile the oracle restatement (FP contraction off: float32 IEEE order)."""
    cmd = ["g++", "-std=c++17", "-O2", "-march=x86-64-v2", "-mfma", "-ffp-contract=off", "-fPIC", "-shared",
           "-o", ORACLE_SO, os.path.join(HERE, "pt_oracle.cpp"), "-lpthread"]
    if not quiet:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_ref(quiet=True):
    """Build oracle/_ref/libref.so when the reference checkout is present."""
    if not os.path.isdir(REF_SRC):
        return None
    from importlib import util
    spec = util.spec_from_file_location("build_ref", os.path.join(HERE, "build_ref.py"))
    mod = util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(REF_SRC, quiet=quiet)


def require_fma():
    """The oracle and the reference build use the CPU's fused multiply-add
    instruction (the triangle test; -mfma, nothing else contracted): fail
    clearly on a CPU without it rather than on an illegal instruction."""
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return
    if " fma" not in flags:
        raise RuntimeError("the CPU oracle needs a CPU with fused multiply-add (x86 FMA3)")


def _f(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _u(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_uint32))


class Oracle:
    """The C++ restatement (pt_oracle.cpp)."""

    def __init__(self, pt):
        require_fma()
        src = os.path.join(HERE, "pt_oracle.cpp")
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(src) > os.path.getmtime(ORACLE_SO):
            build_oracle()
        self.pt = pt
        L = C.CDLL(ORACLE_SO)
        P, F, U, S = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_size_t
        M = C.POINTER(pt.pt_material)
        L.or_scene_create.argtypes = [C.POINTER(pt.pt_scene_desc)]
        L.or_scene_create.restype = P
        L.or_scene_destroy.argtypes = [P]
        L.or_scene_materials.argtypes = [P, M]
        L.or_scene_emitter_cdf.argtypes = [P, F]
        L.or_scene_emitter_cdf.restype = C.c_uint32
        L.or_env_cdf.argtypes = [P, F, F]
        L.or_env_sample.argtypes = [P, C.c_uint32, F, S, F, F, F]
        L.or_env_pdf.argtypes = [P, C.c_uint32, F, S, F, F]
        L.or_rng_batch.argtypes = [C.c_uint32, U, U, S, C.c_uint32, C.c_uint32, C.c_uint32, F]
        L.or_bsdf_eval.argtypes = [C.c_int, M, U, F, F, F, S, F, F]
        L.or_bsdf_sample.argtypes = [C.c_int, M, U, F, F, F, S, F, F, F]
        L.or_phase_sample.argtypes = [C.c_int, F, F, F, S, F, F]
        L.or_lbvh.argtypes = [P, U, U, C.POINTER(C.c_int32)]
        L.or_trace_closest.argtypes = [P, F, S, C.POINTER(pt.pt_hit)]
        L.or_trace_shadow.argtypes = [P, F, S, U, F]
        L.or_render.argtypes = [P, C.POINTER(pt.pt_render_params), F, F, C.c_int, C.POINTER(C.c_uint64)]
        L.or_render.restype = C.c_int
        L.or_render_cached.argtypes = [P, C.POINTER(pt.pt_render_params), F, F, C.c_int, F, C.c_float]
        L.or_render_cached.restype = C.c_int
        self.L = L
        self.h = None
        self.scene = None

    def load(self, scene):
        if self.h:
            self.L.or_scene_destroy(self.h)
        self.scene = scene
        self.h = self.L.or_scene_create(C.byref(scene.desc()))

    def __del__(self):
        try:
            if self.h:
                self.L.or_scene_destroy(self.h)
        except Exception:
            pass

    def materials(self):
        n = len(self.scene.materials)
        out = (self.pt.pt_material * n)()
        self.L.or_scene_materials(self.h, out)
        return out

    def emitter_cdf(self):
        n = self.L.or_scene_emitter_cdf(self.h, None)
        a = np.zeros(n, np.float32)
        self.L.or_scene_emitter_cdf(self.h, _f(a))
        return a

    def env_cdf(self):
        H, W = self.scene.env_rgb.shape[:2]
        m = np.zeros(H + 1, np.float32)
        c = np.zeros(H * (W + 1), np.float32)
        self.L.or_env_cdf(self.h, _f(m), _f(c))
        return m, c

    def env_sample(self, mode, u):
        n = len(u)
        d, r, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.or_env_sample(self.h, mode, _f(u), n, _f(d), _f(r), _f(p))
        return d, r, p

    def env_pdf(self, mode, dirs):
        n = len(dirs)
        p, r = np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        self.L.or_env_pdf(self.h, mode, _f(dirs), n, _f(p), _f(r))
        return p, r

    def rng(self, kind, pixel_ids, sample_ids, dims, w, h):
        out = np.zeros((len(pixel_ids), dims), np.float32)
        self.L.or_rng_batch(kind, _u(pixel_ids), _u(sample_ids), len(pixel_ids), dims, w, h, _f(out))
        return out

    def bsdf_eval(self, mats, mi, wi, wo, h=None, fp64=False):
        n = len(wi)
        ma = (self.pt.pt_material * len(mats))(*mats)
        f, p = np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.or_bsdf_eval(1 if fp64 else 0, ma, _u(mi), _f(wi), _f(wo), _f(h), n, _f(f), _f(p))
        return f, p

    def bsdf_sample(self, mats, mi, wi, u, h=None, fp64=False):
        n = len(wi)
        ma = (self.pt.pt_material * len(mats))(*mats)
        wo, wt, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.or_bsdf_sample(1 if fp64 else 0, ma, _u(mi), _f(wi), _f(u), _f(h), n, _f(wo), _f(wt), _f(p))
        return wo, wt, p

    def phase_sample(self, g, wo, u, fp64=False):
        n = len(wo)
        wi, p = np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.or_phase_sample(1 if fp64 else 0, _f(g), _f(wo), _f(u), n, _f(wi), _f(p))
        return wi, p

    def lbvh(self):
        n = self.scene.num_triangles
        morton, order = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        nodes = np.zeros((max(n - 1, 1), 2), np.int32)
        self.L.or_lbvh(self.h, _u(morton), _u(order), nodes.ctypes.data_as(C.POINTER(C.c_int32)))
        return morton, order, nodes[: max(n - 1, 0)]

    def trace_closest(self, rays):
        n = len(rays)
        out = (self.pt.pt_hit * n)()
        self.L.or_trace_closest(self.h, _f(rays), n, out)
        return np.frombuffer(out, dtype=np.dtype([("t", "<f4"), ("mesh", "<u4"), ("prim", "<u4"), ("u", "<f4"),
                                                  ("v", "<f4"), ("hit", "<u4")]), count=n).copy()

    def trace_shadow(self, rays):
        n = len(rays)
        occ, tr = np.zeros(n, np.uint32), np.zeros((n, 3), np.float32)
        self.L.or_trace_shadow(self.h, _f(rays), n, _u(occ), _f(tr))
        return occ, tr

    def render(self, params, per_path=False, threads=0):
        W, H = params.width, params.height
        s = np.zeros((H, W, 4), np.float32)
        pp = np.zeros((params.spp, H, W, 3), np.float32) if per_path else None
        cnt = (C.c_uint64 * 2)()
        rc = self.L.or_render(self.h, C.byref(params), _f(s), _f(pp), threads, cnt)
        if rc != 0:
            raise RuntimeError("oracle: unsupported scene")
        return s, pp, (cnt[0], cnt[1])

    def render_cached(self, params, value, rough_threshold=0.3, per_path=False, threads=0):
        """Render with paths ended into a constant radiance cache."""
        W, H = params.width, params.height
        s = np.zeros((H, W, 4), np.float32)
        pp = np.zeros((params.spp, H, W, 3), np.float32) if per_path else None
        v = np.asarray(value, np.float32)
        rc = self.L.or_render_cached(self.h, C.byref(params), _f(s), _f(pp), threads, _f(v), rough_threshold)
        if rc != 0:
            raise RuntimeError("oracle: unsupported scene")
        return s, pp


class Reference:
    """The reference's shader code compiled for the CPU (oracle/_ref/libref.so).

    One scene at a time per process (the shader's resources are globals)."""

    def __init__(self, pt, ris=False):
        so = REF_RIS_SO if ris else REF_SO
        if not os.path.exists(so):
            raise FileNotFoundError(so)
        require_fma()
        self.pt = pt
        L = C.CDLL(so)
        F, U, S = C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_size_t
        M = C.POINTER(pt.pt_material)
        L.ref_scene_create.argtypes = [C.POINTER(pt.pt_scene_desc)]
        L.ref_render.argtypes = [C.POINTER(pt.pt_render_params), F, C.c_int]
        L.ref_scene_materials.argtypes = [M]
        L.ref_rng.argtypes = [U, U, S, C.c_uint32, C.c_uint32, C.c_uint32, F]
        L.ref_bsdf_eval.argtypes = [M, U, F, F, F, S, F, F]
        L.ref_bsdf_sample.argtypes = [M, U, F, F, U, U, C.c_uint32, C.c_uint32, C.c_uint32, S, F, F, F]
        L.ref_hg_sample.argtypes = [F, F, U, U, C.c_uint32, C.c_uint32, C.c_uint32, S, F, F]
        L.ref_env_sample.argtypes = [F, S, F, F, F]
        L.ref_env_pdf.argtypes = [F, S, F, F]
        L.ref_env_cdf.argtypes = [F, F]
        self.L = L
        self.scene = None

    @staticmethod
    def available(ris=False):
        return os.path.exists(REF_RIS_SO if ris else REF_SO)

    def load(self, scene):
        self.scene = scene
        rc = self.L.ref_scene_create(C.byref(scene.desc()))
        if rc != 0:
            raise RuntimeError("reference: scene setup failed")

    def materials(self):
        n = len(self.scene.materials)
        out = (self.pt.pt_material * n)()
        self.L.ref_scene_materials(out)
        return out

    def render(self, params, threads=0):
        W, H = params.width, params.height
        s = np.zeros((H, W, 4), np.float32)
        rc = self.L.ref_render(C.byref(params), _f(s), threads)
        if rc != 0:
            raise RuntimeError(f"reference render rejected parameters ({rc})")
        return s

    def rng(self, pixel_ids, sample_ids, dims, w, h):
        out = np.zeros((len(pixel_ids), dims), np.float32)
        self.L.ref_rng(_u(pixel_ids), _u(sample_ids), len(pixel_ids), dims, w, h, _f(out))
        return out

    def bsdf_eval(self, mats, mi, wi, wo, h=None):
        n = len(wi)
        ma = (self.pt.pt_material * len(mats))(*mats)
        f, p = np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.ref_bsdf_eval(ma, _u(mi), _f(wi), _f(wo), _f(h), n, _f(f), _f(p))
        return f, p

    def bsdf_sample(self, mats, mi, wi, h, pix, smp, dim0, w, hh):
        n = len(wi)
        ma = (self.pt.pt_material * len(mats))(*mats)
        wo, wt, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.ref_bsdf_sample(ma, _u(mi), _f(wi), _f(h), _u(pix), _u(smp), dim0, w, hh, n, _f(wo), _f(wt), _f(p))
        return wo, wt, p

    def hg_sample(self, g, wo, pix, smp, dim0, w, h):
        n = len(wo)
        wi, p = np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.ref_hg_sample(_f(g), _f(wo), _u(pix), _u(smp), dim0, w, h, n, _f(wi), _f(p))
        return wi, p

    def env_sample(self, u):
        n = len(u)
        d, r, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self.L.ref_env_sample(_f(u), n, _f(d), _f(r), _f(p))
        return d, r, p

    def env_pdf(self, dirs):
        n = len(dirs)
        p, r = np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        self.L.ref_env_pdf(_f(dirs), n, _f(p), _f(r))
        return p, r

    def env_cdf(self):
        H, W = self.scene.env_rgb.shape[:2]
        m = np.zeros(H + 1, np.float32)
        c = np.zeros(H * (W + 1), np.float32)
        self.L.ref_env_cdf(_f(m), _f(c))
        return m, c
