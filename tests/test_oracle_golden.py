"""The oracle against the golden values of the reference's validation suite
(tests/golden/furnace.json, generated by tests/golden/make_golden.py):

* Disney lobe furnaces: whole-image mean within +-2 % of the Mitsuba 3
  reference means (validation_tests/disney, pass band of its README);
* volume Beer-Lambert: exp(-2) +- 0.01; volume white furnace: 1 +- 0.04
  (validation_tests/volumetric_tests);
* hair white furnace: the Chiang BCSDF of shaders/Hair.hlsli with
  sigma_a = 0; the FP64 quadrature of f |cos| over the sphere (converged:
  doubling the grid changes it by < 1e-5) is 0.9971 - 0.9999 over incident
  angles and fibre offsets, i.e. the reference's model loses up to 0.3 % of
  the energy (cuticle tilt + trimmed-logistic approximations).  The test
  holds it to 1 within 3e-3.
"""

import json
import os

import numpy as np
import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "furnace.json")))


def furnace_scene(pt, scenes, lobe, W=64):
    g = GOLDEN["disney_furnace"][lobe]
    p = g["params"]
    v, f = scenes.icosphere(4)
    if g["bsdf_type"] == "disney":
        m = pt.make_material(pt.PT_MAT_DISNEY, tuple(p.get("baseColor", [0.8, 0.8, 0.8])))
        for k in ("roughness", "metallic", "specular", "specularTint", "sheen", "sheenTint", "subsurface",
                  "clearcoat", "clearcoatGloss", "anisotropic"):
            if k in p:
                setattr(m, k, p[k])
    else:
        m = pt.make_material(pt.PT_MAT_DIFFUSE, tuple(p.get("albedo", [0.5, 0.5, 0.5])))
    m.vertexOffset, m.vertexCount, m.indexOffset, m.indexCount = 0, len(v), 0, f.size
    env = np.ones((2, 4, 3), np.float32)
    sc = pt.Scene(v, f, [m], normals=v, env_rgb=env)
    cam = scenes.look_at_camera((0, 0, 4), (0, 0, 0), (0, 1, 0), g["fov"], 1.0)
    return sc, cam, g


@pytest.mark.parametrize("lobe", ["diffuse", "metallic_smooth", "metallic_rough", "clearcoat", "lambertian"])
def test_disney_furnace(lobe, pt, scenes, oracle):
    sc, cam, g = furnace_scene(pt, scenes, lobe)
    oracle.load(sc)
    P = pt.render_params(64, 64, 32, cam, max_depth=32)
    s, _, _ = oracle.render(P)
    img = s[..., :3] / s[..., 3:4]
    mean = float(img.mean())
    ref = g["mitsuba_image_mean"]
    assert abs(mean / ref - 1.0) < g["tolerance_rel"], (lobe, mean, ref)


def volume_scene(pt, scenes, name):
    g = GOLDEN["volume"][name]
    p = g["params"]
    tri = np.array([[1000, 1000, -1000], [1001, 1000, -1000], [1000, 1001, -1000]], np.float32)
    m = pt.make_material(pt.PT_MAT_DIFFUSE, (0.5, 0.5, 0.5))
    m.vertexCount, m.indexCount = 3, 3
    vol = pt.pt_volume()
    vol.vmin[:] = p["boundsMin"]
    vol.vmax[:] = p["boundsMax"]
    vol.sigma_a[:] = [p["sigmaA"]] * 3
    vol.sigma_s[:] = [p["sigmaS"]] * 3
    vol.phase_g = p["g"]
    vol.flags = 0
    vol.density_grid = pt.PT_NO_TEXTURE
    sc = pt.Scene(tri, np.array([0, 1, 2]), [m], env_rgb=np.ones((2, 4, 3), np.float32), volumes=[vol])
    cam_z = 3.0 if name == "beer_lambert" else 8.0
    cam = scenes.look_at_camera((0, 0, cam_z), (0, 0, 0), (0, 1, 0), g["fov"], 1.0)
    return sc, cam, g


@pytest.mark.parametrize("name", ["beer_lambert", "white_furnace"])
def test_volume_golden(name, pt, scenes, oracle):
    sc, cam, g = volume_scene(pt, scenes, name)
    oracle.load(sc)
    P = pt.render_params(32, 32, 64, cam, max_depth=32)
    s, _, _ = oracle.render(P)
    mean = float((s[..., :3] / s[..., 3:4]).mean())
    assert abs(mean - g["expected"]) < g["tolerance_abs"], (name, mean)


def hair_furnace_integral(pt, oracle, h, n_theta=400, n_phi=800, theta_i=0.3):
    """FP64 midpoint quadrature of f(wi, wo) |wo.z| over the sphere of wo,
    for the hair frame of shaders/Hair.hlsli (x = tangent, sin(theta) = w.x)."""
    m = pt.make_material(pt.PT_MAT_HAIR, (1.0, 1.0, 1.0))
    m.roughness, m.betaN, m.alpha, m.intIOR = 0.3, 0.3, 2.0, 1.55
    th = (np.arange(n_theta) + 0.5) / n_theta * np.pi - np.pi / 2
    ph = (np.arange(n_phi) + 0.5) / n_phi * 2 * np.pi - np.pi
    T, Ph = np.meshgrid(th, ph, indexing="ij")
    wo = np.stack([np.sin(T), np.cos(T) * np.cos(Ph), np.cos(T) * np.sin(Ph)], -1).reshape(-1, 3).astype(np.float32)
    wi = np.tile(np.array([np.sin(theta_i), np.cos(theta_i) * np.cos(0.7), np.cos(theta_i) * np.sin(0.7)],
                          np.float32), (len(wo), 1))
    hh = np.full(len(wo), h, np.float32)
    f, _ = oracle.bsdf_eval([m], None, wi, wo, hh, fp64=True)
    integrand = f[:, 1].astype(np.float64) * np.abs(wo[:, 2])
    dA = (np.pi / n_theta) * (2 * np.pi / n_phi) * np.cos(T).reshape(-1)
    return float((integrand * dA).sum())


@pytest.mark.parametrize("h", [-0.6, -0.2, 0.0, 0.3, 0.7])
@pytest.mark.parametrize("theta_i", [0.0, 0.8, 1.2])
def test_hair_white_furnace(h, theta_i, pt, oracle):
    e = hair_furnace_integral(pt, oracle, h, theta_i=theta_i)
    assert abs(e - 1.0) < 3e-3, e
