"""EXR output of the host (host/exr.cpp), the EXR/PFM reader and the
comparison tool (compare.py, the statistics of the reference's
validation_tests/compare_exr.py), and the reference's Disney furnace
validation run end to end: XML scene -> nori_render -> EXR -> compare."""

import ctypes as C
import importlib
import importlib.util
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from test_nori_host import LIBNORI, nori, write_hdr, write_obj  # noqa: F401  (nori: fixture)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pbrt-renderer-_b200")
CLI = os.path.join(PKG, "host", "nori_render")
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "furnace.json")))
from oracle.oracle import REF_ROOT  # noqa: E402

REF_DISNEY = os.path.join(REF_ROOT, "validation_tests", "disney")


def _mod(name):
    spec = importlib.util.spec_from_file_location("pbrt_b200_" + name, os.path.join(PKG, name + ".py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


imageio = _mod("imageio")
compare = _mod("compare")


def _writer():
    L = C.CDLL(LIBNORI)
    L.nori_write_exr.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_char_p, C.c_size_t]
    return L.nori_write_exr


def write_exr(path, img):
    err = C.create_string_buffer(256)
    a = np.ascontiguousarray(img, np.float32)
    assert _writer()(str(path).encode(), a.shape[1], a.shape[0], a.ctypes.data, err, 256) == 0, err.value


def test_exr_round_trip_exact(tmp_path):
    rng = np.random.default_rng(0)
    img = (rng.standard_normal((37, 53, 3)) * 10.0).astype(np.float32)
    img[0, 0] = [np.inf, 0.0, -0.0]
    p = tmp_path / "a.exr"
    write_exr(p, img)
    back = imageio.read_exr(str(p))
    assert back.shape == img.shape and np.array_equal(back, img)


def test_exr_is_readable_by_opencv(tmp_path):
    """An independent OpenEXR decoder reads the host's file to the same floats."""
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(1)
    img = rng.uniform(0, 50, (24, 31, 3)).astype(np.float32)
    p = tmp_path / "b.exr"
    write_exr(p, img)
    raw = cv2.imread(str(p), cv2.IMREAD_UNCHANGED | cv2.IMREAD_ANYDEPTH)
    assert raw is not None and raw.dtype == np.float32
    assert np.array_equal(raw[..., ::-1], img)


def test_exr_writer_rejects_bad_arguments(tmp_path):
    w = _writer()
    err = C.create_string_buffer(256)
    assert w(str(tmp_path / "x.exr").encode(), 0, 4, None, err, 256) == -1
    assert b"empty image" in err.value
    px = np.zeros((2, 2, 3), np.float32)
    assert w(str(tmp_path / "no" / "dir.exr").encode(), 2, 2, px.ctypes.data, err, 256) == -1


@pytest.mark.skipif(not os.path.isdir(REF_DISNEY), reason="reference checkout not present")
@pytest.mark.parametrize("lobe", ["diffuse", "clearcoat"])
def test_reads_the_reference_mitsuba_exr(lobe):
    """The reference's Mitsuba renders (compressed EXR) read to the image means
    recorded in the golden fixture."""
    pytest.importorskip("cv2")
    img = imageio.read_exr(os.path.join(REF_DISNEY, f"ref_furnace_{lobe}.exr"))
    assert abs(float(img.mean()) - GOLDEN["disney_furnace"][lobe]["mitsuba_image_mean"]) < 1e-6


def test_compare_statistics():
    rng = np.random.default_rng(2)
    ref = rng.uniform(0.1, 2.0, (16, 16, 3)).astype(np.float32)
    r = compare.compare(ref, ref)
    assert r["relmse"] == 0.0 and r["rmse"] == 0.0 and r["tonemap_psnr_db"] == float("inf")
    ours = ref * 1.1
    r = compare.compare(ours, ref)
    expect = float((((ours.astype(np.float64) - ref) ** 2) / (ref.astype(np.float64) ** 2 + 1e-2)).mean())
    assert abs(r["relmse"] - expect) < 1e-12
    assert all(abs(c["ratio"] - 1.1) < 1e-5 for c in r["channels"].values())
    with pytest.raises(ValueError):
        compare.compare(ref, ref[:8])


def test_compare_cli_json(tmp_path):
    write_exr(tmp_path / "a.exr", np.full((8, 8, 3), 2.0, np.float32))
    write_exr(tmp_path / "b.exr", np.full((8, 8, 3), 1.0, np.float32))
    out = subprocess.run([sys.executable, os.path.join(PKG, "compare.py"), str(tmp_path / "a.exr"),
                          str(tmp_path / "b.exr"), "--json"], capture_output=True, text=True, check=True).stdout
    r = json.loads(out)
    assert abs(r["relmse"] - 1.0 / 1.01) < 1e-9 and abs(r["channels"]["G"]["ratio"] - 2.0) < 1e-12


def furnace_xml(d, lobe, W=128, spp=64):
    """The reference's furnace_<lobe>.xml setup (camera at (0, 0, 4), fov 45,
    a unit sphere, white envmap at the scene's default path) with the BSDF
    parameters recorded in the golden fixture; the sphere is this suite's own
    mesh."""
    from conftest import load_package

    load_package()
    scenes = importlib.import_module("pbrt_b200.scenes")
    g = GOLDEN["disney_furnace"][lobe]
    v, f = scenes.icosphere(4)
    write_obj(d / "sphere.obj", v, f, with_normals=True)
    (d / "textures").mkdir(exist_ok=True)
    write_hdr(d / "textures" / "white_furnace.hdr", np.ones((2, 2, 3), np.float32))
    if g["bsdf_type"] == "disney":
        props = "".join(f'<color name="{k}" value="{" ".join(map(str, val))}"/>' if isinstance(val, list)
                        else f'<float name="{k}" value="{val}"/>' for k, val in g["params"].items())
        bsdf = f'<bsdf type="disney">{props}</bsdf>'
    else:
        albedo = " ".join(map(str, g["params"]["albedo"]))
        bsdf = f'<bsdf type="diffuse"><color name="albedo" value="{albedo}"/></bsdf>'
    (d / "scene.xml").write_text(f"""<scene>
  <integrator type="path_mis"/>
  <camera type="perspective"><float name="fov" value="{g['fov']}"/>
    <transform name="toWorld"><lookat target="0, 0, 0" origin="0, 0, 4" up="0, 1, 0"/></transform>
    <integer name="height" value="{W}"/><integer name="width" value="{W}"/></camera>
  <sampler type="independent"><integer name="sampleCount" value="{spp}"/></sampler>
  <mesh type="obj"><string name="filename" value="sphere.obj"/>{bsdf}</mesh>
</scene>""")
    return g


def test_furnace_xml_loads(nori, tmp_path):
    furnace_xml(tmp_path, "clearcoat")
    from test_nori_host import load

    h, err = load(nori, tmp_path / "scene.xml")
    assert h, err
    nori.nori_free(h)


@pytest.mark.gpu
@pytest.mark.parametrize("lobe", ["diffuse", "metallic_rough", "clearcoat", "lambertian"])
def test_furnace_validation_end_to_end(lobe, tmp_path):
    """validation_tests/disney flow: render the XML with the CLI to an EXR and
    compare its image mean with Mitsuba's (the reference's pass band: 2 %)."""
    g = furnace_xml(tmp_path, lobe)
    out = tmp_path / "ours.exr"
    r = subprocess.run([CLI, str(tmp_path / "scene.xml"), "64", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = imageio.read_exr(str(out))
    assert img.shape == (128, 128, 3) and np.isfinite(img).all()
    mean = float(img.mean())
    assert abs(mean / g["mitsuba_image_mean"] - 1.0) < g["tolerance_rel"], (lobe, mean)
