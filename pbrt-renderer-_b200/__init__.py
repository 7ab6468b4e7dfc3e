"""Python binding of libpt (include/pt.h) — the sm_100a wavefront path tracer.

This package directory holds the CUDA library (csrc/), the C++17 Nori host
(host/) and this ctypes binding, which bench.py and the tests use.  The
binding loads ``csrc/libpt.so`` from this directory and raises if it is
missing: there is no CPU fallback.

Because the directory name is not a Python identifier, load it with
``load_package()`` from a file path (see bench.py), which registers it as
``pbrt_b200``.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPT_PATH = os.path.join(HERE, "csrc", "libpt.so")

PT_OK = 0
PT_MAT_DIFFUSE, PT_MAT_MIRROR, PT_MAT_DIELECTRIC, PT_MAT_MICROFACET, PT_MAT_DISNEY, PT_MAT_HAIR, PT_MAT_SUBSURFACE = range(7)
PT_NO_TEXTURE = 0xFFFFFFFF
PT_VOLUME_HETEROGENEOUS = 1
PT_RNG_SOBOL_OWEN, PT_RNG_PCG_HASH = 0, 1
PT_ENV_CDF, PT_ENV_ALIAS = 0, 1
PT_MEM_HOST, PT_MEM_DEVICE = 0, 1
PT_SAMPLE_DIMS = 4
PT_RENDER_STAGE_TIMING = 1
PT_RENDER_RADIANCE_CACHE = 2
PT_RENDER_RIS_NEE = 4
PT_RENDER_MEDIA_WAVEFRONT = 8
PT_CACHE_PARAMS = 21504
PT_CACHE_FEATURES = 64
PT_CACHE_RECORD_FLOATS = 16
PT_CACHE_MAX_RECORDS = 262144
PT_CACHE_NO_TRAIN = 1
PT_DEBUG_SHADOW_QUEUE_CAP, PT_DEBUG_CACHE_STALL, PT_DEBUG_TAIL, PT_DEBUG_WIDE_PLAN = 1, 2, 3, 4
PT_E_DEVICE = -5


class pt_material(C.Structure):
    """GPUMaterial of the reference (shaders/Common.hlsli:55-89), 144 bytes."""
    _fields_ = [
        ("type", C.c_uint32), ("albedo", C.c_float * 3), ("intIOR", C.c_float), ("extIOR", C.c_float),
        ("alpha", C.c_float), ("isEmitter", C.c_uint32), ("radiance", C.c_float * 3),
        ("indexOffset", C.c_uint32), ("vertexOffset", C.c_uint32), ("indexCount", C.c_uint32),
        ("vertexCount", C.c_uint32), ("surfaceArea", C.c_float), ("emitterCdfOffset", C.c_uint32),
        ("albedoTexIndex", C.c_uint32), ("normalTexIndex", C.c_uint32), ("roughnessTexIndex", C.c_uint32),
        ("metallicTexIndex", C.c_uint32), ("specularTexIndex", C.c_uint32), ("subsurfaceTexIndex", C.c_uint32),
        ("alphaTexIndex", C.c_uint32), ("roughness", C.c_float), ("metallic", C.c_float), ("specular", C.c_float),
        ("specularTint", C.c_float), ("sheen", C.c_float), ("sheenTint", C.c_float), ("subsurface", C.c_float),
        ("clearcoat", C.c_float), ("clearcoatGloss", C.c_float), ("anisotropic", C.c_float), ("betaN", C.c_float),
        ("emitterSelectionProb", C.c_float),
    ]


assert C.sizeof(pt_material) == 144


class pt_volume(C.Structure):
    _fields_ = [("vmin", C.c_float * 3), ("vmax", C.c_float * 3), ("sigma_a", C.c_float * 3),
                ("sigma_s", C.c_float * 3), ("phase_g", C.c_float), ("flags", C.c_uint32),
                ("density_grid", C.c_uint32)]


class pt_grid(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("d", C.c_uint32), ("data", C.POINTER(C.c_float))]


class pt_texture(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("rgba8", C.POINTER(C.c_uint8)), ("srgb", C.c_uint32)]


class pt_scene_desc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint32), ("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
        ("texcoords", C.POINTER(C.c_float)), ("tangents", C.POINTER(C.c_float)),
        ("num_indices", C.c_uint32), ("indices", C.POINTER(C.c_uint32)),
        ("num_meshes", C.c_uint32), ("materials", C.POINTER(pt_material)),
        ("env_width", C.c_uint32), ("env_height", C.c_uint32), ("env_rgb", C.POINTER(C.c_float)),
        ("env_scale", C.c_float), ("ev_compensation", C.c_float),
        ("num_volumes", C.c_uint32), ("volumes", C.POINTER(pt_volume)),
        ("num_grids", C.c_uint32), ("grids", C.POINTER(pt_grid)),
        ("num_textures", C.c_uint32), ("textures", C.POINTER(pt_texture)),
    ]


class pt_camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("llc", C.c_float * 3), ("horizontal", C.c_float * 3),
                ("vertical", C.c_float * 3), ("lens_radius", C.c_float), ("focal_distance", C.c_float)]


class pt_render_params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("sample_offset", C.c_uint32), ("max_depth", C.c_uint32), ("rng_kind", C.c_uint32),
                ("env_sampling", C.c_uint32), ("wave_paths", C.c_uint32), ("flags", C.c_uint32),
                ("camera", pt_camera)]


class pt_film(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("sum", C.c_void_p), ("comp", C.c_void_p),
                ("location", C.c_uint32)]


class pt_stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("waves", C.c_uint64), ("bounces", C.c_uint64), ("launches", C.c_uint64), ("ms_total", C.c_float),
                ("ms_raygen", C.c_float), ("ms_extend", C.c_float), ("ms_shade", C.c_float),
                ("ms_shadow", C.c_float), ("ms_film", C.c_float), ("ms_cache", C.c_float), ("ms_tail", C.c_float),
                ("tail_extension_rays", C.c_uint64)]


class pt_hit(C.Structure):
    _fields_ = [("t", C.c_float), ("mesh", C.c_uint32), ("prim", C.c_uint32), ("u", C.c_float),
                ("v", C.c_float), ("hit", C.c_uint32)]


class pt_request(C.Structure):
    _fields_ = [("params", pt_render_params), ("film", pt_film)]


class pt_batch_tuning(C.Structure):
    _fields_ = [("wave_paths", C.c_uint32), ("traversal_grid", C.c_float), ("ms", C.c_float),
                ("candidates", C.c_uint32), ("candidate_ms", C.c_float * 16), ("candidate_wave", C.c_uint32 * 16),
                ("candidate_grid", C.c_float * 16)]


class pt_cache_params(C.Structure):
    _fields_ = [("train_records", C.c_uint32), ("unbiased_every", C.c_uint32), ("rough_threshold", C.c_float),
                ("learning_rate", C.c_float), ("ema", C.c_float), ("seed", C.c_uint32), ("flags", C.c_uint32),
                ("bbox_min", C.c_float * 3), ("bbox_max", C.c_float * 3), ("max_train_fraction", C.c_float)]


class pt_cache_stats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("last_records", C.c_uint32), ("last_loss", C.c_float),
                ("queries", C.c_uint64), ("last_kernel_ms", C.c_float), ("last_render_infer_ms", C.c_float),
                ("last_render_train_ms", C.c_float), ("last_render_train_rows", C.c_uint64)]


def cache_params(train_records=0, unbiased_every=0, rough_threshold=0.0, learning_rate=0.0, ema=0.0, seed=0,
                 flags=0, bbox=None, max_train_fraction=0.0) -> pt_cache_params:
    p = pt_cache_params()
    p.max_train_fraction = max_train_fraction
    p.train_records, p.unbiased_every, p.rough_threshold = train_records, unbiased_every, rough_threshold
    p.learning_rate, p.ema, p.seed, p.flags = learning_rate, ema, seed, flags
    if bbox is not None:
        p.bbox_min[:] = bbox[0]
        p.bbox_max[:] = bbox[1]
    return p


def fptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def uptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_uint32))


def vptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Scene:
    """Flattened scene arrays (the buffers CreateSceneBuffers uploads) + pt_scene_desc."""

    def __init__(self, positions, indices, materials, normals=None, texcoords=None, tangents=None,
                 env_rgb=None, env_scale=1.0, ev_compensation=0.0, volumes=(), grids=(), textures=()):
        """textures: (H, W, 4) uint8 RGBA arrays, or (array, srgb) pairs (srgb
        defaults to False); materials refer to them by index."""
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        nv = len(self.positions)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(nv, 3)
        self.texcoords = None if texcoords is None else np.ascontiguousarray(texcoords, np.float32).reshape(nv, 2)
        self.tangents = None if tangents is None else np.ascontiguousarray(tangents, np.float32).reshape(nv, 3)
        self.materials = (pt_material * len(materials))(*materials)
        if env_rgb is None:
            env_rgb = np.zeros((1, 1, 3), np.float32)
        self.env_rgb = np.ascontiguousarray(env_rgb, np.float32)
        self.env_scale = float(env_scale)
        self.ev_compensation = float(ev_compensation)
        self.volumes = (pt_volume * max(1, len(volumes)))(*volumes)
        self.num_volumes = len(volumes)
        self.grid_arrays = [np.ascontiguousarray(g, np.float32) for g in grids]
        gl = [pt_grid(g.shape[2], g.shape[1], g.shape[0], fptr(g)) for g in self.grid_arrays]
        self.grids = (pt_grid * max(1, len(gl)))(*gl)
        self.tex_arrays, self.tex_srgb, tl = [], [], []
        for t in textures:
            img, srgb = (t if isinstance(t, tuple) else (t, False))
            self.tex_srgb.append(bool(srgb))
            img = np.ascontiguousarray(img, np.uint8)
            if img.ndim != 3 or img.shape[2] != 4:
                raise ValueError("textures are (H, W, 4) uint8 RGBA arrays")
            self.tex_arrays.append(img)
            tl.append(pt_texture(img.shape[1], img.shape[0], img.ctypes.data_as(C.POINTER(C.c_uint8)), int(srgb)))
        self.textures = (pt_texture * max(1, len(tl)))(*tl)

    @property
    def num_triangles(self):
        return len(self.indices) // 3

    def desc(self) -> pt_scene_desc:
        d = pt_scene_desc()
        d.num_vertices = len(self.positions)
        d.positions = fptr(self.positions)
        d.normals = fptr(self.normals)
        d.texcoords = fptr(self.texcoords)
        d.tangents = fptr(self.tangents)
        d.num_indices = len(self.indices)
        d.indices = uptr(self.indices)
        d.num_meshes = len(self.materials)
        d.materials = C.cast(self.materials, C.POINTER(pt_material))
        d.env_height, d.env_width = self.env_rgb.shape[0], self.env_rgb.shape[1]
        d.env_rgb = fptr(self.env_rgb)
        d.env_scale = self.env_scale
        d.ev_compensation = self.ev_compensation
        d.num_volumes = self.num_volumes
        d.volumes = C.cast(self.volumes, C.POINTER(pt_volume))
        d.num_grids = len(self.grid_arrays)
        d.grids = C.cast(self.grids, C.POINTER(pt_grid))
        d.num_textures = len(self.tex_arrays)
        d.textures = C.cast(self.textures, C.POINTER(pt_texture))
        self._desc = d
        return d


def make_material(type=PT_MAT_DIFFUSE, albedo=(0.5, 0.5, 0.5), **kw) -> pt_material:
    """A pt_material with the reference's BSDFGPUData defaults (include/bsdf.h:58-88)."""
    m = pt_material()
    m.type = type
    m.albedo[:] = albedo
    m.intIOR, m.extIOR, m.alpha = 1.5046, 1.000277, 0.1
    m.roughness, m.metallic, m.specular, m.specularTint = 0.5, 0.0, 0.5, 0.0
    m.sheen, m.sheenTint, m.subsurface, m.clearcoat = 0.0, 0.5, 0.0, 0.0
    m.clearcoatGloss, m.anisotropic, m.betaN = 1.0, 0.0, 0.3
    for f in ("albedoTexIndex", "normalTexIndex", "roughnessTexIndex", "metallicTexIndex", "specularTexIndex",
              "subsurfaceTexIndex", "alphaTexIndex"):
        setattr(m, f, PT_NO_TEXTURE)
    for k, v in kw.items():
        if k == "radiance":
            m.radiance[:] = v
            m.isEmitter = 1
        else:
            setattr(m, k, v)
    return m


def render_params(width, height, spp, camera: pt_camera, max_depth=32, sample_offset=0,
                  rng_kind=PT_RNG_SOBOL_OWEN, env_sampling=PT_ENV_CDF, wave_paths=0, flags=0) -> pt_render_params:
    p = pt_render_params()
    p.width, p.height, p.spp, p.sample_offset = width, height, spp, sample_offset
    p.max_depth, p.rng_kind, p.env_sampling, p.wave_paths = max_depth, rng_kind, env_sampling, wave_paths
    p.flags = flags
    p.camera = camera
    return p


class PTError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libpt.so (built by __graft_entry__.build()); raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPT_PATH):
            raise PTError(f"libpt.so not built: {LIBPT_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIBPT_PATH)
        P, F, U, S = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_size_t
        L.pt_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
        L.pt_destroy.argtypes = [P]
        L.pt_set_stream.argtypes = [P, C.c_void_p]
        L.pt_debug_set.argtypes = [P, C.c_uint32, C.c_uint64]
        L.pt_last_error.argtypes = [P]
        L.pt_last_error.restype = C.c_char_p
        L.pt_upload_scene.argtypes = [P, C.POINTER(pt_scene_desc)]
        L.pt_render.argtypes = [P, C.POINTER(pt_render_params), C.POINTER(pt_film), C.POINTER(pt_stats)]
        L.pt_bsdf_eval_batch.argtypes = [P, C.POINTER(pt_material), C.c_uint32, U, F, F, F, S, F, F, C.c_uint32]
        L.pt_bsdf_sample_batch.argtypes = [P, C.POINTER(pt_material), C.c_uint32, U, F, F, F, S, F, F, F, C.c_uint32]
        L.pt_phase_sample_batch.argtypes = [P, F, F, F, S, F, F, C.c_uint32]
        L.pt_env_sample_batch.argtypes = [P, C.c_uint32, F, S, F, F, F, C.c_uint32]
        L.pt_env_pdf_batch.argtypes = [P, C.c_uint32, F, S, F, F, C.c_uint32]
        L.pt_env_read_cdf.argtypes = [P, F, F]
        L.pt_rng_batch.argtypes = [P, C.c_uint32, U, U, S, C.c_uint32, C.c_uint32, C.c_uint32, F, C.c_uint32]
        L.pt_bvh_info.argtypes = [P, U, U]
        L.pt_bvh_read.argtypes = [P, U, U, C.POINTER(C.c_int32)]
        L.pt_trace_closest.argtypes = [P, F, S, C.POINTER(pt_hit), C.c_uint32]
        L.pt_trace_shadow.argtypes = [P, F, S, U, F, C.c_uint32]
        L.pt_render_batch.argtypes = [P, C.POINTER(pt_request), C.c_uint32, F, C.POINTER(pt_stats)]
        L.pt_batch_autotune.argtypes = [P, C.POINTER(pt_request), C.c_uint32, C.POINTER(pt_batch_tuning)]
        L.pt_cache_init.argtypes = [P, C.POINTER(pt_cache_params)]
        L.pt_cache_release.argtypes = [P]
        L.pt_cache_weights.argtypes = [P, F, F]
        L.pt_cache_encode_batch.argtypes = [P, F, S, F, C.c_uint32]
        L.pt_cache_infer_batch.argtypes = [P, F, S, F, C.c_uint32]
        L.pt_cache_gradient_batch.argtypes = [P, F, F, S, F, F, C.c_uint32]
        L.pt_cache_train_batch.argtypes = [P, F, F, S, F, C.c_uint32]
        L.pt_cache_get_stats.argtypes = [P, C.POINTER(pt_cache_stats)]
        _lib = L
    return _lib


class Context:
    """One pt_ctx: a CUDA stream on `device` and one uploaded scene."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.pt_create(C.byref(h), device)
        if rc != 0:
            raise PTError(f"pt_create failed ({rc})")
        self.h = h
        self.scene = None

    def _check(self, rc):
        if rc != 0:
            raise PTError(f"libpt error {rc}: {self.L.pt_last_error(self.h).decode()}")

    def debug_set(self, what, value):
        """Test hooks of the device error paths (pt_debug_set)."""
        self._check(self.L.pt_debug_set(self.h, what, value))

    def set_stream(self, stream_ptr):
        """Run libpt work on an existing CUDA stream (an int cudaStream_t)."""
        self._check(self.L.pt_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def close(self):
        if self.h:
            self.L.pt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, scene: Scene):
        self.scene = scene
        self._check(self.L.pt_upload_scene(self.h, C.byref(scene.desc())))

    def render(self, params: pt_render_params, film_sum=None, film_comp=None, location=PT_MEM_HOST):
        W, H = params.width, params.height
        if location == PT_MEM_HOST:
            if film_sum is None:
                film_sum = np.zeros((H, W, 4), np.float32)
            if film_comp is None:
                film_comp = np.zeros((H, W, 4), np.float32)
            film = pt_film(W, H, film_sum.ctypes.data, film_comp.ctypes.data, PT_MEM_HOST)
        else:  # device pointers (ints), e.g. torch tensors' data_ptr()
            film = pt_film(W, H, film_sum, film_comp, PT_MEM_DEVICE)
        st = pt_stats()
        self._check(self.L.pt_render(self.h, C.byref(params), C.byref(film), C.byref(st)))
        return film_sum, film_comp, st

    def bsdf_eval(self, mats, mat_index, wi, wo, h=None):
        n = len(wi)
        ma = (pt_material * len(mats))(*mats)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.L.pt_bsdf_eval_batch(self.h, ma, len(mats), uptr(mat_index), fptr(wi), fptr(wo),
                                              fptr(h), n, fptr(f), fptr(pdf), PT_MEM_HOST))
        return f, pdf

    def bsdf_sample(self, mats, mat_index, wi, u, h=None):
        n = len(wi)
        ma = (pt_material * len(mats))(*mats)
        wo = np.zeros((n, 3), np.float32)
        wt = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.L.pt_bsdf_sample_batch(self.h, ma, len(mats), uptr(mat_index), fptr(wi), fptr(u), fptr(h),
                                                n, fptr(wo), fptr(wt), fptr(pdf), PT_MEM_HOST))
        return wo, wt, pdf

    def phase_sample(self, g, wo, u):
        n = len(wo)
        wi = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.L.pt_phase_sample_batch(self.h, fptr(g), fptr(wo), fptr(u), n, fptr(wi), fptr(pdf),
                                                 PT_MEM_HOST))
        return wi, pdf

    def env_sample(self, mode, u):
        n = len(u)
        d = np.zeros((n, 3), np.float32)
        r = np.zeros((n, 3), np.float32)
        p = np.zeros(n, np.float32)
        self._check(self.L.pt_env_sample_batch(self.h, mode, fptr(u), n, fptr(d), fptr(r), fptr(p), PT_MEM_HOST))
        return d, r, p

    def env_pdf(self, mode, dirs):
        n = len(dirs)
        p = np.zeros(n, np.float32)
        r = np.zeros((n, 3), np.float32)
        self._check(self.L.pt_env_pdf_batch(self.h, mode, fptr(dirs), n, fptr(p), fptr(r), PT_MEM_HOST))
        return p, r

    def env_cdf(self):
        s = self.scene
        H, W = s.env_rgb.shape[0], s.env_rgb.shape[1]
        marg = np.zeros(H + 1, np.float32)
        cond = np.zeros(H * (W + 1), np.float32)
        self._check(self.L.pt_env_read_cdf(self.h, fptr(marg), fptr(cond)))
        return marg, cond

    def rng(self, kind, pixel_ids, sample_ids, dims, width, height):
        n = len(pixel_ids)
        out = np.zeros((n, dims), np.float32)
        self._check(self.L.pt_rng_batch(self.h, kind, uptr(pixel_ids), uptr(sample_ids), n, dims, width, height,
                                        fptr(out), PT_MEM_HOST))
        return out

    def bvh(self):
        nt, nw = C.c_uint32(), C.c_uint32()
        self._check(self.L.pt_bvh_info(self.h, C.byref(nt), C.byref(nw)))
        n = nt.value
        morton = np.zeros(n, np.uint32)
        order = np.zeros(n, np.uint32)
        nodes = np.zeros((max(n - 1, 1), 2), np.int32)
        self._check(self.L.pt_bvh_read(self.h, uptr(morton), uptr(order),
                                       nodes.ctypes.data_as(C.POINTER(C.c_int32))))
        return morton, order, nodes[: max(n - 1, 0)], nw.value

    def trace_closest(self, rays):
        n = len(rays)
        out = (pt_hit * n)()
        self._check(self.L.pt_trace_closest(self.h, fptr(rays), n, out, PT_MEM_HOST))
        a = np.frombuffer(out, dtype=np.dtype([("t", "<f4"), ("mesh", "<u4"), ("prim", "<u4"), ("u", "<f4"),
                                               ("v", "<f4"), ("hit", "<u4")]), count=n).copy()
        return a

    def trace_shadow(self, rays):
        n = len(rays)
        occ = np.zeros(n, np.uint32)
        tr = np.zeros((n, 3), np.float32)
        self._check(self.L.pt_trace_shadow(self.h, fptr(rays), n, uptr(occ), fptr(tr), PT_MEM_HOST))
        return occ, tr

    # ---- batched requests ------------------------------------------------------------
    @staticmethod
    def _requests(params_list, films, location):
        n = len(params_list)
        reqs = (pt_request * n)()
        for i, (p, f) in enumerate(zip(params_list, films)):
            reqs[i].params = p
            if location == PT_MEM_HOST:
                reqs[i].film = pt_film(p.width, p.height, f[0].ctypes.data, f[1].ctypes.data, PT_MEM_HOST)
            else:
                reqs[i].film = pt_film(p.width, p.height, f[0], f[1], PT_MEM_DEVICE)
        return reqs

    def render_batch(self, params_list, films=None, location=PT_MEM_HOST):
        """Render several requests in one batch.  films: per request (sum, comp)
        host arrays (H, W, 4) or device pointers; None = fresh host films.
        Returns (films, per-request ms, stats)."""
        if films is None:
            films = [(np.zeros((p.height, p.width, 4), np.float32), np.zeros((p.height, p.width, 4), np.float32))
                     for p in params_list]
        reqs = self._requests(params_list, films, location)
        ms = np.zeros(len(params_list), np.float32)
        st = pt_stats()
        self._check(self.L.pt_render_batch(self.h, reqs, len(params_list), fptr(ms), C.byref(st)))
        return films, ms, st

    def batch_autotune(self, params_list, films=None, location=PT_MEM_HOST) -> pt_batch_tuning:
        if films is None:
            films = [(np.zeros((p.height, p.width, 4), np.float32), np.zeros((p.height, p.width, 4), np.float32))
                     for p in params_list]
        reqs = self._requests(params_list, films, location)
        out = pt_batch_tuning()
        self._check(self.L.pt_batch_autotune(self.h, reqs, len(params_list), C.byref(out)))
        return out

    # ---- radiance cache ------------------------------------------------------------
    def cache_init(self, params: pt_cache_params | None = None):
        self._check(self.L.pt_cache_init(self.h, C.byref(params if params is not None else cache_params())))

    def cache_release(self):
        self._check(self.L.pt_cache_release(self.h))

    def cache_weights(self, set_to=None):
        """The FP32 parameters (PT_CACHE_PARAMS); with set_to, replace them first."""
        if set_to is not None:
            w = np.ascontiguousarray(set_to, np.float32)
            assert w.size == PT_CACHE_PARAMS
            self._check(self.L.pt_cache_weights(self.h, None, fptr(w)))
        out = np.zeros(PT_CACHE_PARAMS, np.float32)
        self._check(self.L.pt_cache_weights(self.h, fptr(out), None))
        return out

    def cache_encode(self, records):
        r = np.ascontiguousarray(records, np.float32).reshape(-1, PT_CACHE_RECORD_FLOATS)
        out = np.zeros((len(r), PT_CACHE_FEATURES), np.float32)
        self._check(self.L.pt_cache_encode_batch(self.h, fptr(r), len(r), fptr(out), PT_MEM_HOST))
        return out

    def cache_infer(self, features):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, PT_CACHE_FEATURES)
        out = np.zeros((len(f), 3), np.float32)
        self._check(self.L.pt_cache_infer_batch(self.h, fptr(f), len(f), fptr(out), PT_MEM_HOST))
        return out

    def cache_gradient(self, features, targets):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, PT_CACHE_FEATURES)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        g = np.zeros(PT_CACHE_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self.L.pt_cache_gradient_batch(self.h, fptr(f), fptr(t), len(f), fptr(g), fptr(loss),
                                                   PT_MEM_HOST))
        return g, float(loss[0])

    def cache_train(self, features, targets):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, PT_CACHE_FEATURES)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        loss = np.zeros(1, np.float32)
        self._check(self.L.pt_cache_train_batch(self.h, fptr(f), fptr(t), len(f), fptr(loss), PT_MEM_HOST))
        return float(loss[0])

    def cache_stats(self) -> pt_cache_stats:
        st = pt_cache_stats()
        self._check(self.L.pt_cache_get_stats(self.h, C.byref(st)))
        return st
