"""Seeded synthetic workloads for the path tracer.

The reference measures on its own scene files, whose large assets are absent
(envmaps, hair, density grids); these generators stand in for them with the
shapes, sizes and value distributions of the benchmark configurations:

* ``cornell``        — 12-triangle room + icosphere (subdiv 3, 1280 tris,
                       Disney roughness 0.5) + one quad light of radiance 17.
* ``disney_spheres`` — n x n UV spheres of 20,480 triangles each with Disney
                       parameters drawn U[0,1] (roughness U[0.05,1]) and a
                       procedural sky + sun HDR envmap (peak 5e4).
* ``hair_volume``    — camera-facing hair ribbons (Chiang BCSDF) inside an
                       fBm density grid (heterogeneous medium).

Every array is float32 / uint32 and every draw comes from
``numpy.random.default_rng(seed)``.
"""

from __future__ import annotations

import copy
import math

import numpy as np

from . import (PT_MAT_DIFFUSE, PT_MAT_DISNEY, PT_MAT_HAIR, PT_MAT_SUBSURFACE, PT_NO_TEXTURE,
               PT_VOLUME_HETEROGENEOUS, Scene, make_material, pt_camera, pt_volume)


# ---------------------------------------------------------------------------
# camera: the lower-left-corner / image-plane form of CameraConstants
# (src/gpu/DXRApp_Camera.cpp:84-112) from a look-at and a vertical fov.
# ---------------------------------------------------------------------------
def look_at_camera(origin, target, up, fov_y_deg, aspect, lens_radius=0.0, focal_distance=1.0) -> pt_camera:
    o = np.asarray(origin, np.float64)
    f = np.asarray(target, np.float64) - o
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    half_h = math.tan(math.radians(fov_y_deg) * 0.5)
    half_w = half_h * aspect
    llc = o + f - half_w * r - half_h * u
    c = pt_camera()
    c.pos[:] = o.astype(np.float32)
    c.llc[:] = llc.astype(np.float32)
    c.horizontal[:] = (2 * half_w * r).astype(np.float32)
    c.vertical[:] = (2 * half_h * u).astype(np.float32)
    c.lens_radius = lens_radius
    c.focal_distance = focal_distance
    return c


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                cache[k] = len(v) - 1
            return cache[k]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v, np.float64), np.array(f, np.uint32)


def uv_sphere(slices: int, rings: int):
    """UV sphere with 2 * slices * (rings - 1) triangles (pole fans + quads)."""
    verts = [(0.0, 1.0, 0.0)]
    for i in range(1, rings):
        th = math.pi * i / rings
        for j in range(slices):
            ph = 2 * math.pi * j / slices
            verts.append((math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph)))
    verts.append((0.0, -1.0, 0.0))
    v = np.array(verts, np.float64)
    bot = len(verts) - 1
    faces = []
    ring = lambda i, j: 1 + (i - 1) * slices + (j % slices)
    for j in range(slices):
        faces.append((0, ring(1, j + 1), ring(1, j)))
    for i in range(1, rings - 1):
        for j in range(slices):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            faces.append((a, b, d))
            faces.append((a, d, c))
    for j in range(slices):
        faces.append((bot, ring(rings - 1, j), ring(rings - 1, j + 1)))
    return v, np.array(faces, np.uint32)


class _Builder:
    def __init__(self):
        self.pos, self.nrm, self.uv, self.tan, self.idx, self.mats = [], [], [], [], [], []
        self.nv = 0
        self.ni = 0

    def add(self, pos, faces, mat, normals=None, uvs=None, tangents=None):
        pos = np.asarray(pos, np.float32)
        faces = np.asarray(faces, np.uint32).reshape(-1)
        mat.vertexOffset, mat.vertexCount = self.nv, len(pos)
        mat.indexOffset, mat.indexCount = self.ni, len(faces)
        self.pos.append(pos)
        self.nrm.append(np.zeros_like(pos) if normals is None else np.asarray(normals, np.float32))
        self.uv.append(np.zeros((len(pos), 2), np.float32) if uvs is None else np.asarray(uvs, np.float32))
        self.tan.append(np.zeros_like(pos) if tangents is None else np.asarray(tangents, np.float32))
        self.idx.append(faces)
        self.mats.append(mat)
        self.nv += len(pos)
        self.ni += len(faces)

    def scene(self, **kw) -> Scene:
        return Scene(np.concatenate(self.pos), np.concatenate(self.idx), self.mats, normals=np.concatenate(self.nrm),
                     texcoords=np.concatenate(self.uv), tangents=np.concatenate(self.tan), **kw)


def _quad(p0, p1, p2, p3):
    return np.array([p0, p1, p2, p3], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def _flat_normals(pos, faces):
    p = np.asarray(pos, np.float64)
    f = np.asarray(faces).reshape(-1, 3)
    n = np.cross(p[f[0, 1]] - p[f[0, 0]], p[f[0, 2]] - p[f[0, 0]])
    n /= np.linalg.norm(n)
    return np.tile(n.astype(np.float32), (len(p), 1))


# ---------------------------------------------------------------------------
# configuration 1: Cornell-style box
# ---------------------------------------------------------------------------
def cornell(width=256, height=256, subdiv=3, many_lights=False):
    """Closed 12-triangle room (white 0.73, red 0.65, green 0.12 walls), a Disney
    icosphere (roughness 0.5) and a downward quad light of radiance 17."""
    b = _Builder()
    white = make_material(PT_MAT_DIFFUSE, (0.73, 0.73, 0.73))
    red = make_material(PT_MAT_DIFFUSE, (0.65, 0.05, 0.05))
    green = make_material(PT_MAT_DIFFUSE, (0.12, 0.45, 0.15))
    # room x in [-1,1], y in [0,2], z in [-1,1]; faces wound to face inward
    walls_w = []
    walls_w.append(_quad((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1)))    # floor (+y)
    walls_w.append(_quad((-1, 2, -1), (-1, 2, 1), (1, 2, 1), (1, 2, -1)))    # ceiling (-y)
    walls_w.append(_quad((-1, 0, -1), (-1, 2, -1), (1, 2, -1), (1, 0, -1)))  # back (+z)
    walls_w.append(_quad((-1, 0, 1), (1, 0, 1), (1, 2, 1), (-1, 2, 1)))      # front (-z)
    pw = np.concatenate([w[0] for w in walls_w])
    fw = np.concatenate([w[1] + 4 * i for i, w in enumerate(walls_w)])
    nw = np.concatenate([_flat_normals(w[0], w[1]) for w in walls_w])
    b.add(pw, fw, white, normals=nw)
    pl, fl = _quad((-1, 0, -1), (-1, 0, 1), (-1, 2, 1), (-1, 2, -1))       # left (+x), red
    b.add(pl, fl, red, normals=_flat_normals(pl, fl))
    pr, fr = _quad((1, 0, -1), (1, 2, -1), (1, 2, 1), (1, 0, 1))           # right (-x), green
    b.add(pr, fr, green, normals=_flat_normals(pr, fr))
    # light: 0.5 x 0.5 quad just under the ceiling, normal -y (or four small
    # coloured quads of uneven power, for many-light sampling)
    y = 1.98
    if not many_lights:
        pq, fq = _quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25))
        light = make_material(PT_MAT_DIFFUSE, (0.0, 0.0, 0.0), radiance=(17.0, 17.0, 17.0))
        b.add(pq, fq, light, normals=_flat_normals(pq, fq))
    else:
        for (cx, cz, s, rad) in ((-0.6, -0.6, 0.12, (40.0, 8.0, 8.0)), (0.6, -0.5, 0.2, (6.0, 20.0, 6.0)),
                                 (0.0, 0.5, 0.3, (4.0, 4.0, 12.0)), (0.55, 0.55, 0.08, (90.0, 90.0, 60.0))):
            pq, fq = _quad((cx - s, y, cz - s), (cx + s, y, cz - s), (cx + s, y, cz + s), (cx - s, y, cz + s))
            light = make_material(PT_MAT_DIFFUSE, (0.0, 0.0, 0.0), radiance=rad)
            b.add(pq, fq, light, normals=_flat_normals(pq, fq))
    v, f = icosphere(subdiv)
    sph = make_material(PT_MAT_DISNEY, (0.8, 0.6, 0.4), roughness=0.5)
    c, r = np.array([0.0, 0.55, -0.1]), 0.55
    b.add(v * r + c, f, sph, normals=v)
    scene = b.scene()
    cam = look_at_camera((0.0, 1.0, 0.95), (0.0, 0.9, -1.0), (0, 1, 0), 62.0, width / height)
    return scene, cam


def subsurface_scene(width=64, height=64, subdiv=3, mfp=0.08, g=0.2):
    """The Cornell room with its sphere made of a subsurface material (type 6:
    rough dielectric boundary over a scattering interior; mean free path
    `mfp`, HG anisotropy `g`, tint (1, 0.9, 0.8) in sheen / sheenTint /
    clearcoat as the reference stores it)."""
    sc, cam = cornell(width, height, subdiv)
    mats = [copy.copy(m) for m in sc.materials]
    m = mats[-1]
    m.type = PT_MAT_SUBSURFACE
    m.albedo[:] = (0.9, 0.55, 0.45)
    m.roughness, m.specular = 0.3, 0.5
    m.sheen, m.sheenTint, m.clearcoat = 1.0, 0.9, 0.8
    m.subsurface, m.anisotropic = mfp, g
    m.intIOR, m.extIOR = 1.4, 1.0
    return Scene(sc.positions, sc.indices, mats, normals=sc.normals, texcoords=sc.texcoords,
                 tangents=sc.tangents), cam


# ---------------------------------------------------------------------------
# textured materials: every map the shading reads, plus an alpha cut-out
# ---------------------------------------------------------------------------
def texture_maps(seed=0):
    """Seeded procedural RGBA8 maps: (albedo checker [sRGB], bump normal map,
    roughness ramp, specular noise, floor albedo [sRGB], soft circular alpha)."""
    rng = np.random.default_rng(seed)
    n = 64
    y, x = np.mgrid[0:n, 0:n]
    check = ((x // 8 + y // 8) % 2)[..., None]
    albedo = np.where(check, [200, 60, 40, 255], [40, 90, 200, 255]).astype(np.uint8)
    hx, hy = np.sin(x / n * 8 * math.pi), np.cos(y / n * 6 * math.pi)
    nv = np.stack([-0.4 * hx, -0.4 * hy, np.ones_like(hx)], -1)
    nv /= np.linalg.norm(nv, axis=-1, keepdims=True)
    normal = np.concatenate([np.clip(np.rint((nv * 0.5 + 0.5) * 255), 0, 255), np.full((n, n, 1), 255)], -1)
    rough = np.zeros((16, 16, 4), np.uint8)
    rough[..., 0] = np.linspace(25, 230, 16, dtype=np.uint8)[None, :]
    rough[..., 3] = 255
    spec = rng.integers(0, 256, (8, 8, 4)).astype(np.uint8)
    spec[..., 3] = 255
    floor = rng.integers(60, 220, (128, 128, 4)).astype(np.uint8)
    floor[..., 3] = 255
    r = np.hypot(x - n / 2 + 0.5, y - n / 2 + 0.5) / (n / 2)
    a = np.clip((1.0 - r) * 3.0, 0, 1)
    alpha = np.stack([a * 255, a * 180, a * 120, a * 255], -1)
    return [(albedo, True), normal.astype(np.uint8), rough, spec, (floor, True),
            np.clip(np.rint(alpha), 0, 255).astype(np.uint8)]


def textured_scene(width=96, height=72, seed=0, slices=48, rings=25, maps=None):
    """A Disney sphere with albedo / normal / roughness / specular maps, a
    floor with a tiled albedo map (UVs up to 4, wrap addressing), an
    alpha-cut quad between them and a small area light under a dim sky."""
    b = _Builder()
    maps = texture_maps(seed) if maps is None else maps
    v, f = uv_sphere(slices, rings)
    uv = np.stack([np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi) + 0.5, np.arccos(np.clip(v[:, 1], -1, 1)) / math.pi], 1)
    sph = make_material(PT_MAT_DISNEY, (0.8, 0.8, 0.8), roughness=0.5, metallic=0.1, clearcoat=0.3)
    sph.albedoTexIndex, sph.normalTexIndex, sph.roughnessTexIndex, sph.specularTexIndex = 0, 1, 2, 3
    b.add(v * 0.8 + np.array([0.0, 0.0, 0.0]), f, sph, normals=v, uvs=uv)
    fl = make_material(PT_MAT_DIFFUSE, (0.7, 0.7, 0.7))
    fl.albedoTexIndex = 4
    fp, ff = _quad((-3, -0.8, -3), (-3, -0.8, 3), (3, -0.8, 3), (3, -0.8, -3))
    b.add(fp, ff, fl, normals=_flat_normals(fp, ff), uvs=[(0, 0), (0, 4), (4, 4), (4, 0)])
    cut = make_material(PT_MAT_DIFFUSE, (0.3, 0.8, 0.3))
    cut.alphaTexIndex = 5
    cp, cf = _quad((-0.6, -0.6, 1.2), (0.6, -0.6, 1.2), (0.6, 0.6, 1.2), (-0.6, 0.6, 1.2))
    b.add(cp, cf, cut, normals=_flat_normals(cp, cf), uvs=[(0, 1), (1, 1), (1, 0), (0, 0)])
    light = make_material(PT_MAT_DIFFUSE, (0.0, 0.0, 0.0), radiance=(12.0, 12.0, 12.0))
    lp, lf = _quad((-0.5, 2.5, 1.5), (0.5, 2.5, 1.5), (0.5, 2.5, 2.5), (-0.5, 2.5, 2.5))
    b.add(lp, lf, light, normals=_flat_normals(lp, lf))
    scene = b.scene(env_rgb=sky_envmap(64, 32, sun_peak=30.0), env_scale=0.3, textures=maps)
    cam = look_at_camera((0.4, 0.6, 3.2), (0.0, -0.1, 0.0), (0, 1, 0), 45.0, width / height)
    return scene, cam


# ---------------------------------------------------------------------------
# configuration 2: Disney sphere grid under a procedural sky
# ---------------------------------------------------------------------------
def sky_envmap(width=2048, height=1024, sun_peak=5.0e4, sun_elev_deg=35.0, sun_azim_deg=60.0, sun_sigma_deg=0.6):
    """Equirectangular RGB float32 envmap (row 0 = zenith, y-up convention of
    shaders/Envmap.hlsli:15-24): sky gradient above the horizon, dark ground
    below, and a Gaussian sun lobe of the given peak radiance."""
    y = (np.arange(height) + 0.5) / height
    x = (np.arange(width) + 0.5) / width
    theta = np.pi * y[:, None]
    phi = 2 * np.pi * x[None, :]
    d = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta) * np.ones_like(phi), np.sin(theta) * np.sin(phi)], -1)
    up = np.clip(d[..., 1], -1, 1)
    zen = np.array([0.25, 0.45, 1.0])
    hor = np.array([1.0, 0.95, 0.9])
    gnd = np.array([0.12, 0.10, 0.08])
    t = np.clip(up, 0, 1)[..., None] ** 0.5
    sky = hor * (1 - t) + zen * t
    env = np.where(up[..., None] > 0, sky * 1.5, gnd)
    el, az = math.radians(sun_elev_deg), math.radians(sun_azim_deg)
    s = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    ang = np.arccos(np.clip((d * s).sum(-1), -1, 1))
    sig = math.radians(sun_sigma_deg)
    env = env + sun_peak * np.exp(-0.5 * (ang / sig) ** 2)[..., None] * np.array([1.0, 0.95, 0.85])
    return env.astype(np.float32)


def disney_spheres(width=1280, height=720, grid=8, slices=128, rings=81, seed=0, env_w=2048, env_h=1024):
    rng = np.random.default_rng(seed)
    b = _Builder()
    v, f = uv_sphere(slices, rings)
    spacing = 2.5
    off = (grid - 1) * spacing / 2
    for i in range(grid):
        for j in range(grid):
            m = make_material(PT_MAT_DISNEY, tuple(rng.uniform(0, 1, 3)))
            m.roughness = float(rng.uniform(0.05, 1.0))
            m.metallic, m.specular, m.specularTint = (float(x) for x in rng.uniform(0, 1, 3))
            m.sheen, m.sheenTint, m.subsurface = (float(x) for x in rng.uniform(0, 1, 3))
            m.clearcoat, m.clearcoatGloss = (float(x) for x in rng.uniform(0, 1, 2))
            c = np.array([i * spacing - off, 1.0, j * spacing - off])
            b.add(v + c, f, m, normals=v)
    env = sky_envmap(env_w, env_h)
    scene = b.scene(env_rgb=env, env_scale=1.0)
    ext = off + 2.0
    cam = look_at_camera((0.0, 1.15 * ext + 3.0, 1.6 * ext + 4.0), (0.0, 0.5, 0.0), (0, 1, 0), 40.0, width / height)
    return scene, cam


# ---------------------------------------------------------------------------
# configuration 3: hair ribbons in a heterogeneous medium
# ---------------------------------------------------------------------------
def eumelanin_to_color(eu, beta_n):
    """Colour whose Chiang-Eq.-9 inversion (shaders/Hair.hlsli:125-133) gives the
    PBRT eumelanin absorption sigma_a = eu * (0.419, 0.697, 1.37)."""
    sa = eu * np.array([0.419, 0.697, 1.37])
    bn = beta_n
    den = 5.969 - 0.215 * bn + 2.532 * bn ** 2 - 10.73 * bn ** 3 + 5.574 * bn ** 4 + 0.245 * bn ** 5
    return np.exp(-np.sqrt(sa) * den)


def fbm_grid(n=128, seed=0, octaves=5):
    rng = np.random.default_rng(seed)
    out = np.zeros((n, n, n), np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        r = 4 * 2 ** o
        lat = rng.uniform(0, 1, (r + 1, r + 1, r + 1))
        c = np.linspace(0, r, n, endpoint=False) + 0.5 * r / n
        i0 = np.floor(c).astype(int)
        t = c - i0
        i0 = np.clip(i0, 0, r - 1)
        t = t * t * (3 - 2 * t)

        def interp(a, ax):
            a0 = np.take(a, i0, axis=ax)
            a1 = np.take(a, i0 + 1, axis=ax)
            sh = [1, 1, 1]
            sh[ax] = n
            tt = t.reshape(sh)
            return a0 * (1 - tt) + a1 * tt

        out += amp * interp(interp(interp(lat, 0), 1), 2)
        total += amp
        amp *= 0.5
    out /= total
    # sphere falloff + contrast, density in [0, 1]
    g = (np.arange(n) + 0.5) / n * 2 - 1
    rr = np.sqrt(g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2)
    d = np.clip((out - 0.45) * 3.0, 0, 1) * np.clip(1.2 - rr, 0, 1)
    return d.astype(np.float32)


def hair_volume(width=1024, height=1024, strands=20000, segments=32, seed=0, grid_n=128, g=0.3):
    rng = np.random.default_rng(seed)
    b = _Builder()
    cam_pos = np.array([0.0, 0.0, 4.0])
    # strands: roots on a unit sphere cap, gently curved downward
    roots = rng.normal(size=(strands, 3))
    roots /= np.linalg.norm(roots, axis=1, keepdims=True)
    roots[:, 1] = np.abs(roots[:, 1])
    length = rng.uniform(0.6, 1.2, strands)
    width_h = 0.004
    eu = rng.uniform(0.1, 8.0, strands)
    s = np.linspace(0, 1, segments + 1)
    ribbons_pos, ribbons_uv, ribbons_tan, faces = [], [], [], []
    # one mesh per eumelanin band keeps the material count small
    bands = 8
    band_of = np.minimum((eu - 0.1) / (7.9 / bands), bands - 1).astype(int)
    for band in range(bands):
        ids = np.nonzero(band_of == band)[0]
        if len(ids) == 0:
            continue
        P, UV, T, F = [], [], [], []
        nv = 0
        for k in ids:
            r0 = roots[k]
            out = r0 + np.array([0, -0.3, 0])
            pts = r0[None, :] + (s[:, None] * length[k]) * (out / np.linalg.norm(out))[None, :]
            pts[:, 1] -= 0.5 * (s * length[k]) ** 2
            tang = np.gradient(pts, axis=0)
            tang /= np.linalg.norm(tang, axis=1, keepdims=True)
            view = cam_pos[None, :] - pts
            side = np.cross(tang, view)
            side /= np.linalg.norm(side, axis=1, keepdims=True) + 1e-12
            left, right = pts - side * width_h, pts + side * width_h
            for i in range(segments + 1):
                P += [left[i], right[i]]
                UV += [(s[i], 0.0), (s[i], 1.0)]   # UV.y = (h + 1) / 2 across the ribbon
                T += [tang[i], tang[i]]
            for i in range(segments):
                a = nv + 2 * i
                F += [(a, a + 1, a + 3), (a, a + 3, a + 2)]
            nv += 2 * (segments + 1)
        eu_mid = 0.1 + (band + 0.5) * 7.9 / bands
        col = eumelanin_to_color(eu_mid, 0.3)
        m = make_material(PT_MAT_HAIR, tuple(col))
        m.roughness, m.betaN, m.alpha, m.intIOR = 0.3, 0.3, 2.0, 1.55
        b.add(np.array(P), np.array(F), m, uvs=np.array(UV), tangents=np.array(T))
    dens = fbm_grid(grid_n, seed)
    vol = pt_volume()
    vol.vmin[:] = (-1.6, -1.6, -1.6)
    vol.vmax[:] = (1.6, 1.6, 1.6)
    vol.sigma_a[:] = (0.2, 0.2, 0.2)
    vol.sigma_s[:] = (1.8, 1.8, 1.8)   # albedo 0.9
    vol.phase_g = g
    vol.flags = PT_VOLUME_HETEROGENEOUS
    vol.density_grid = 0
    env = sky_envmap(512, 256, sun_peak=2.0e3)
    scene = b.scene(env_rgb=env, volumes=[vol], grids=[dens])
    cam = look_at_camera(tuple(cam_pos), (0, 0.2, 0), (0, 1, 0), 45.0, width / height)
    return scene, cam


# ---------------------------------------------------------------------------
# configuration 5: the radiance-cache scene (~10 M triangles, mixed materials)
# ---------------------------------------------------------------------------
def displaced_icosphere(subdiv, seed, amp=0.12):
    """Icosphere with a smooth radial displacement (a sum of 12 random
    spherical waves); returns positions, faces and vertex normals."""
    v, f = icosphere(subdiv)
    rng = np.random.default_rng(seed)
    k = rng.normal(size=(12, 3))
    k /= np.linalg.norm(k, axis=1, keepdims=True)
    freq = rng.uniform(2.0, 9.0, 12)
    ph = rng.uniform(0, 2 * np.pi, 12)
    w = rng.uniform(0.3, 1.0, 12) / np.arange(1, 13)
    disp = (np.sin((v @ k.T) * freq + ph) * w).sum(1)
    disp = amp * disp / np.abs(disp).max()
    p = v * (1.0 + disp)[:, None]
    tri = p[f]
    fn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n = np.zeros_like(p)
    for c in range(3):
        np.add.at(n, f[:, c], fn)
    n /= np.linalg.norm(n, axis=1, keepdims=True) + 1e-20
    return p, f, n


def radiance_cache_scene(width=1920, height=1080, instances=122, subdiv=6, seed=0, volume=True):
    """Configuration 5: `instances` copies (random scale, rotation, placement)
    of one displaced icosphere of 81,920 triangles (~10 M triangles at 122),
    on a ground plane with a back wall; Disney materials (U[0,1] parameters,
    roughness U[0.05, 1]) with every 7th instance a hair material (BCSDF on
    the sphere surface, h from the UV parametrisation); a homogeneous fog
    box over part of the scene (albedo 0.9, g 0.3) when `volume`; the sky +
    sun envmap at 2048 x 1024."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    base_p, base_f, base_n = displaced_icosphere(subdiv, seed + 1)
    # spherical UVs for hair's h and tangent frame
    base_uv = np.stack([0.5 + np.arctan2(base_p[:, 0], base_p[:, 2]) / (2 * np.pi),
                        0.5 + np.arcsin(np.clip(base_p[:, 1] / np.linalg.norm(base_p, axis=1), -1, 1)) / np.pi], 1)
    side = int(np.ceil(np.sqrt(instances)))
    for i in range(instances):
        gx, gz = i % side, i // side
        s = rng.uniform(0.5, 1.1)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, bq, c, d = q
        R = np.array([[a * a + bq * bq - c * c - d * d, 2 * (bq * c - a * d), 2 * (bq * d + a * c)],
                      [2 * (bq * c + a * d), a * a - bq * bq + c * c - d * d, 2 * (c * d - a * bq)],
                      [2 * (bq * d - a * c), 2 * (c * d + a * bq), a * a - bq * bq - c * c + d * d]])
        t = np.array([(gx - side / 2) * 2.6 + rng.uniform(-0.4, 0.4), s * 1.05,
                      (gz - side / 2) * 2.6 + rng.uniform(-0.4, 0.4)])
        pos = (base_p @ R.T) * s + t
        nrm = base_n @ R.T
        if i % 7 == 3:
            m = make_material(PT_MAT_HAIR, tuple(eumelanin_to_color(rng.uniform(0.3, 4.0), 0.3)))
            m.roughness, m.betaN, m.alpha, m.intIOR = 0.3, 0.3, 2.0, 1.55
        else:
            m = make_material(PT_MAT_DISNEY, tuple(rng.uniform(0, 1, 3)))
            m.roughness = float(rng.uniform(0.05, 1.0))
            m.metallic, m.specular, m.specularTint = (float(x) for x in rng.uniform(0, 1, 3))
            m.sheen, m.sheenTint, m.subsurface = (float(x) for x in rng.uniform(0, 1, 3))
            m.clearcoat, m.clearcoatGloss = (float(x) for x in rng.uniform(0, 1, 2))
        b.add(pos, base_f, m, normals=nrm, uvs=base_uv)
    ext = side * 1.3 + 4
    pg, fg = _quad((-ext, 0, -ext), (-ext, 0, ext), (ext, 0, ext), (ext, 0, -ext))
    ground = make_material(PT_MAT_DISNEY, (0.6, 0.58, 0.55))
    ground.roughness = 0.7
    b.add(pg, fg, ground, normals=_flat_normals(pg, fg))
    pw, fw = _quad((-ext, 0, -ext), (ext, 0, -ext), (ext, 12, -ext), (-ext, 12, -ext))
    wall = make_material(PT_MAT_DIFFUSE, (0.7, 0.7, 0.72))
    b.add(pw, fw, wall, normals=_flat_normals(pw, fw))
    env = sky_envmap(2048, 1024, sun_peak=2.0e4)
    vols = []
    if volume:
        v = pt_volume()
        v.vmin[:] = (-ext * 0.2, 0.0, -ext * 0.6)
        v.vmax[:] = (ext * 0.6, 3.0, ext * 0.3)
        v.sigma_a[:] = (0.003, 0.003, 0.003)
        v.sigma_s[:] = (0.027, 0.027, 0.027)   # albedo 0.9
        v.phase_g = 0.3
        v.flags = 0
        v.density_grid = PT_NO_TEXTURE
        vols.append(v)
    scene = b.scene(env_rgb=env, env_scale=1.0, volumes=vols)
    cam = look_at_camera((0.0, side * 1.1 + 3.0, side * 1.5 + 6.0), (0.0, 0.5, 0.0), (0, 1, 0), 42.0, width / height)
    return scene, cam


def sample_directions(n, seed, upper=False):
    """Uniform unit vectors (upper hemisphere if `upper`), float32."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    if upper:
        d[:, 2] = np.abs(d[:, 2])
    return d.astype(np.float32)


# ---------------------------------------------------------------------------
# configuration 4: batched serving-style requests over the configuration 1-2 scenes
# ---------------------------------------------------------------------------
def batch_requests(n=32, seed=0):
    """n render requests, each on the Cornell box (configuration 1) or the
    Disney spheres (configuration 2) at random: a random camera, image sides
    log-uniform in [64, 1024], spp uniform in {4..256}, the scene's depth
    (8 / 16).  Returns dicts {scene, width, height, spp, max_depth, camera}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        scene = "cornell" if rng.random() < 0.5 else "disney_envmap"
        w = int(round(float(np.exp(rng.uniform(np.log(64), np.log(1024))))))
        h = int(round(float(np.exp(rng.uniform(np.log(64), np.log(1024))))))
        spp = int(rng.integers(4, 257))
        if scene == "cornell":
            eye = (rng.uniform(-0.7, 0.7), rng.uniform(0.3, 1.7), rng.uniform(0.6, 0.95))
            tgt = (rng.uniform(-0.5, 0.5), rng.uniform(0.2, 1.2), rng.uniform(-1.0, -0.2))
            cam = look_at_camera(eye, tgt, (0, 1, 0), float(rng.uniform(40, 70)), w / h)
            depth = 8
        else:
            az, el, dist = rng.uniform(0, 2 * np.pi), np.radians(rng.uniform(15, 50)), rng.uniform(12, 30)
            eye = (dist * np.cos(el) * np.sin(az), 1.0 + dist * np.sin(el), dist * np.cos(el) * np.cos(az))
            tgt = (rng.uniform(-3, 3), 1.0, rng.uniform(-3, 3))
            cam = look_at_camera(eye, tgt, (0, 1, 0), float(rng.uniform(30, 50)), w / h)
            depth = 16
        out.append({"scene": scene, "width": w, "height": h, "spp": spp, "max_depth": depth, "camera": cam})
    return out
