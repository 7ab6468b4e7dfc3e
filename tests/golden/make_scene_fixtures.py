"""Generate the scene and image fixtures of tests/test_reference_scenes.py from
the reference's own scene files and validation images.

Run in a checkout that has the reference mounted (default
$PBRT_REFERENCE_ROOT, else /root/reference) after the Nori host library is
built:

    python tests/golden/make_scene_fixtures.py [--ref <reference checkout>]

Scenes (tests/golden/scenes/<name>.npz): each reference XML is loaded,
unmodified, through this repository's Nori host (XML parser, plugin
registry, OBJ loader, scene flattening, camera conversion) and the
flattened arrays the host would upload are stored: positions, indices,
normals, texcoords, tangents, material records, camera constants, envmap
texels and scale, and the host's scene info.  The GPU tests rebuild the
scene from these arrays, because the reference checkout is not present
where they run; a CPU test re-derives them from the XML whenever the
checkout is present, so a fixture cannot drift from its XML.

Images (tests/golden/images/<name>.npz), both from the reference's
validation suite:
* `mitsuba`: the Mitsuba 3 render the reference validates against
  (linear RGB, stored as float16);
* `dxr_srgb`: the reference's own GPU render of the scene, as its
  comparison tool saved it (diff_*/ours_srgb.png: Reinhard x/(1+x), then
  x^(1/2.2), 8 bit).  The two depth-of-field images are stored as 2x2 block
  means (uint8, 256 x 256) to keep the fixture small.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)

# name -> (scene XML, Mitsuba image, reference GPU render), paths in the reference checkout
SCENES = {
    "cool_scene1": ("scenes/cool_scene1/cornell_box.xml", None, None),
    # the reference's own renders of these two disagree with its Mitsuba
    # images (dof_mitsuba_out.exr, pinhole_mitsuba.exr) by ~20/255 after the
    # tonemap, so only the reference's renders are kept for them
    "dof": ("validation_tests/dof/dof_test_scene.xml", None, "validation_tests/dof/dof_diff/ours_srgb.png"),
    "dof_pinhole": ("validation_tests/dof/dof_pinhole_scene.xml", None,
                    "validation_tests/dof/dof_diff/pinhole_diff/ours_srgb.png"),
    "furnace_ibl": ("validation_tests/ibl_test/sphere_furnace_ibl.xml", "validation_tests/ibl_test/ref_furnace_ibl.exr",
                    "validation_tests/ibl_test/diff_furnace_ibl/ours_srgb.png"),
}
for _lobe in ("diffuse", "metallic_smooth", "metallic_rough", "clearcoat", "lambertian"):
    SCENES["furnace_" + _lobe] = (
        f"validation_tests/disney/furnace_{_lobe}.xml", f"validation_tests/disney/ref_furnace_{_lobe}.exr",
        None if _lobe == "lambertian" else f"validation_tests/disney/diff_furnace_{_lobe}/ours_srgb.png")
BINNED = ("dof", "dof_pinhole")


def flatten(nori, pt, xml):
    """The host's flattened scene as a dict of arrays (see module docstring)."""
    from test_nori_host import scene_from_xml

    sc, cam, info = scene_from_xml(nori, pt, xml)
    empty = np.zeros(0, np.float32)
    return {
        "positions": sc.positions, "indices": sc.indices,
        "normals": empty if sc.normals is None else sc.normals,
        "texcoords": empty if sc.texcoords is None else sc.texcoords,
        "tangents": empty if sc.tangents is None else sc.tangents,
        "materials": np.frombuffer(bytes(sc.materials), np.uint8),
        "camera": np.frombuffer(bytes(cam), np.uint8),
        "env_rgb": sc.env_rgb, "env_scale": np.float32(sc.env_scale),
        "info": np.array(info, np.uint32),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PBRT_REFERENCE_ROOT", "/root/reference"))
    a = ap.parse_args()
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    import cv2

    sys.path.insert(0, TESTS)
    sys.path.insert(0, ROOT)
    from conftest import load_package
    from test_nori_host import nori_lib

    pt = load_package()
    nori = nori_lib()
    os.makedirs(os.path.join(HERE, "scenes"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "images"), exist_ok=True)
    for name, (xml, mitsuba, dxr) in SCENES.items():
        arrays = flatten(nori, pt, os.path.join(a.ref, xml))
        arrays["source"] = np.array(xml)
        np.savez_compressed(os.path.join(HERE, "scenes", name + ".npz"), **arrays)
        img = {}
        if mitsuba:
            m = cv2.imread(os.path.join(a.ref, mitsuba), cv2.IMREAD_UNCHANGED | cv2.IMREAD_ANYDEPTH)
            img["mitsuba"] = m[..., :3][..., ::-1].astype(np.float16)
            img["mitsuba_source"] = np.array(mitsuba)
        if dxr:
            d = cv2.imread(os.path.join(a.ref, dxr), cv2.IMREAD_COLOR)[..., ::-1].astype(np.float64)
            if name in BINNED:
                H, W = d.shape[:2]
                d = d.reshape(H // 2, 2, W // 2, 2, 3).mean((1, 3))
            img["dxr_srgb"] = np.clip(np.round(d), 0, 255).astype(np.uint8)
            img["dxr_binned"] = np.int32(2 if name in BINNED else 1)
            img["dxr_source"] = np.array(dxr)
        if img:
            np.savez_compressed(os.path.join(HERE, "images", name + ".npz"), **img)
        print(name, int(arrays["info"][4]), "triangles", sorted(img))


if __name__ == "__main__":
    main()
