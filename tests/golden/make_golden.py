"""Generate tests/golden/furnace.json from the reference's validation suite.

Run in a checkout that has the reference mounted (default $PBRT_REFERENCE_ROOT,
else /root/reference):

    python tests/golden/make_golden.py [--ref <reference checkout>]

For each Disney furnace scene (validation_tests/disney/furnace_*.xml) it
records the Disney parameters and camera of the XML, and the sphere-masked
mean luminance of the Mitsuba 3 reference image next to it
(ref_furnace_*.exr), computed with the sphere mask of
validation_tests/disney/analyze_furnace.py (unit sphere at the origin, camera
at (0, 0, 4), fov 45).  The pass band (+-2 %) is the one
validation_tests/disney/README.md states.  It also records the volume
Beer-Lambert and white-furnace setups (validation_tests/volumetric_tests)
with their analytic targets.  Only numbers are stored; no reference file is
copied.
"""

from __future__ import annotations

import argparse
import json
import os
import xml.etree.ElementTree as ET

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_xml(path):
    """Parse a Nori scene file; comments are dropped first because some of
    the reference files contain '--' inside comments, which strict XML
    parsers reject."""
    import re
    with open(path, encoding="utf-8") as f:
        text = re.sub(r"<!--.*?-->", "", f.read(), flags=re.S)
    return ET.fromstring(text)


def parse_props(node):
    out = {}
    for ch in node:
        name = ch.get("name")
        if ch.tag == "float":
            out[name] = float(ch.get("value"))
        elif ch.tag == "integer":
            out[name] = int(ch.get("value"))
        elif ch.tag in ("color", "point", "vector"):
            out[name] = [float(x) for x in ch.get("value").replace(",", " ").split()]
        elif ch.tag == "string":
            out[name] = ch.get("value")
    return out


def sphere_mask(W, H, fov_deg=45.0, cam_pos=(0, 0, 4), R=1.0):
    fy = np.tan(np.deg2rad(fov_deg) / 2.0)
    fx = fy * (W / H)
    j, i = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    u = (i + 0.5) / W * 2.0 - 1.0
    v = 1.0 - (j + 0.5) / H * 2.0
    d = np.stack([u * fx, v * fy, -np.ones_like(u)], -1)
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    c = np.array(cam_pos, np.float64)
    b = (d * c).sum(-1)
    return (b * b - (c @ c - R * R)) > 0.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PBRT_REFERENCE_ROOT", "/root/reference"))
    a = ap.parse_args()
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    import cv2

    disney_dir = os.path.join(a.ref, "validation_tests", "disney")
    furnace = {}
    for lobe in ["diffuse", "metallic_smooth", "metallic_rough", "clearcoat", "lambertian"]:
        xml = os.path.join(disney_dir, f"furnace_{lobe}.xml")
        root = load_xml(xml)
        mesh = root.find("mesh")
        bsdf = mesh.find("bsdf")
        cam = root.find("camera")
        cp = parse_props(cam)
        exr = cv2.imread(os.path.join(disney_dir, f"ref_furnace_{lobe}.exr"), cv2.IMREAD_UNCHANGED | cv2.IMREAD_ANYDEPTH)
        img = exr[..., :3][..., ::-1].astype(np.float64)
        H, W = img.shape[:2]
        m = sphere_mask(W, H, cp.get("fov", 45.0))
        px = img[m]
        lum = 0.2126 * px[:, 0] + 0.7152 * px[:, 1] + 0.0722 * px[:, 2]
        furnace[lobe] = {
            "bsdf_type": bsdf.get("type"),
            "params": parse_props(bsdf),
            "fov": cp.get("fov", 45.0),
            "mitsuba_masked_lum_mean": float(lum.mean()),
            "mitsuba_image_mean": float(img.mean()),
            "tolerance_rel": 0.02,
            "source": f"validation_tests/disney/furnace_{lobe}.xml, ref_furnace_{lobe}.exr",
        }
    vol = {}
    for name, rel in [("beer_lambert", "beer_lambert/vol_beer_lambert.xml"),
                      ("white_furnace", "white_furnace/vol_white_furnace.xml")]:
        root = load_xml(os.path.join(a.ref, "validation_tests", "volumetric_tests", rel))
        med = root.find("medium")
        cam = parse_props(root.find("camera"))
        vol[name] = {"medium_type": med.get("type"), "params": parse_props(med), "fov": cam.get("fov"),
                     "width": cam.get("width"), "height": cam.get("height"),
                     "source": f"validation_tests/volumetric_tests/{rel}"}
    vol["beer_lambert"]["expected"] = float(np.exp(-2.0))
    vol["beer_lambert"]["tolerance_abs"] = 0.01
    vol["white_furnace"]["expected"] = 1.0
    vol["white_furnace"]["tolerance_abs"] = 0.04
    out = {"disney_furnace": furnace, "volume": vol,
           "generated_by": "tests/golden/make_golden.py"}
    with open(os.path.join(HERE, "furnace.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1)[:3000])


if __name__ == "__main__":
    main()
