"""Compare two linear HDR renders, as the reference's validation tool does
(validation_tests/compare_exr.py): per-channel means and their ratio, mean
and max absolute difference, linear RMSE, relMSE = mean((x - ref)^2 /
(ref^2 + 1e-2)), and PSNR after a Reinhard + 1/2.2 display curve.

    python pbrt-renderer-_b200/compare.py ours.exr reference.exr [--exposure EV] [--json]
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys

import numpy as np


def reinhard_srgb(img: np.ndarray, exposure_ev: float = 0.0) -> np.ndarray:
    x = np.maximum(img * (2.0 ** exposure_ev), 0.0)
    return np.power(x / (1.0 + x), 1.0 / 2.2)


def relmse(ours: np.ndarray, ref: np.ndarray) -> float:
    return float((((ours - ref) ** 2) / (ref * ref + 1e-2)).mean())


def compare(ours: np.ndarray, ref: np.ndarray, exposure_ev: float = 0.0) -> dict:
    if ours.shape != ref.shape:
        raise ValueError(f"shape mismatch: ours {ours.shape}, reference {ref.shape}")
    ours = ours.astype(np.float64)
    ref = ref.astype(np.float64)
    channels = {}
    for c, name in enumerate("RGB"):
        om, rm = float(ours[..., c].mean()), float(ref[..., c].mean())
        d = np.abs(ours[..., c] - ref[..., c])
        channels[name] = {"ours_mean": om, "ref_mean": rm, "ratio": om / rm if rm > 1e-10 else float("inf"),
                          "mean_abs_diff": float(d.mean()), "max_abs_diff": float(d.max())}
    mse_tm = float(((reinhard_srgb(ours, exposure_ev) - reinhard_srgb(ref, exposure_ev)) ** 2).mean())
    return {"width": int(ours.shape[1]), "height": int(ours.shape[0]), "ours_mean": float(ours.mean()),
            "ref_mean": float(ref.mean()), "channels": channels,
            "rmse": float(np.sqrt(((ours - ref) ** 2).mean())), "relmse": relmse(ours, ref),
            "tonemap_psnr_db": float("inf") if mse_tm <= 1e-10 else 10.0 * np.log10(1.0 / mse_tm)}


def _imageio():
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("pbrt_b200_imageio", os.path.join(here, "imageio.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("ours")
    ap.add_argument("reference")
    ap.add_argument("--exposure", type=float, default=0.0)
    ap.add_argument("--json", action="store_true", help="print the statistics as one JSON object")
    a = ap.parse_args(argv)
    io = _imageio()
    r = compare(io.read_image(a.ours), io.read_image(a.reference), a.exposure)
    if a.json:
        print(json.dumps(r))
        return 0
    print(f"Resolution      : {r['width']} x {r['height']}")
    print(f"{'channel':>8}  {'ours_mean':>10}  {'ref_mean':>10}  {'ratio':>8}  {'mean|diff|':>10}  {'max|diff|':>10}")
    for name, c in r["channels"].items():
        print(f"{name:>8}  {c['ours_mean']:>10.4f}  {c['ref_mean']:>10.4f}  {c['ratio']:>8.4f}  "
              f"{c['mean_abs_diff']:>10.4f}  {c['max_abs_diff']:>10.4f}")
    print(f"Linear RMSE     : {r['rmse']:.5f}")
    print(f"relMSE          : {r['relmse']:.5f}")
    print(f"Tonemap PSNR    : {r['tonemap_psnr_db']:.2f} dB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
