"""Generates tests/golden/camera_ref.npz from the REFERENCE's own camera code.

Runs `ref_harness camera` (oracle/_ref/fp32/ref_harness, built from the reference's sources by
oracle/ref/build_ref.sh; host code only, no GPU needed) on 3DGS cameras.json files and stores,
per file and per settings row, what the viewer's path computes for every camera
(camera_loader.cu:62-90 fromCameraState, main.cu:141-157, camera.cpp:88-156): view and
projection matrices, the six frustum planes, the camera position, the fovy and the resolution.

Inputs:
  * synthetic cameras.json files written by synth.write_cameras_json (regenerated bit for bit
    by the test, so the test needs nothing but the fixture);
  * when the reference tree is present, its own assets/cameras/*.json; those entries carry the
    SHA-256 of the file, and the test compares them only where the same file is present.

Usage (from the repository root):  python tests/golden/make_camera_golden.py
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gaussian-point-splatting_b200"))

import synth  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "fp32", "ref_harness")
REF_ROOT = os.environ.get("GPS_REFERENCE_ROOT", "/root/reference")
MAX_CAMERAS = 40  # the viewer's max_eval_count; keeps the fixture small

# (width, height, fovy, near, far, override_camera_settings): the viewer's defaults, a
# --resolution/--fovy override, and odd sizes that exercise the height rounding
SETTINGS = [
    (1920, 1080, 45.0, 0.2, 10000.0, 0),
    (1280, 720, 60.0, 0.5, 500.0, 1),
    (1001, 333, 30.0, 0.1, 1000.0, 0),
    (777, 555, 75.5, 0.2, 10000.0, 1),
]


def synthetic_json_files(out_dir: str) -> dict[str, str]:
    """The synthetic camera paths: an orbit, random poses inside the town, a tilted portrait
    camera with fx != fy."""
    files = {}
    p = os.path.join(out_dir, "syn_orbit.json")
    synth.write_cameras_json(p, synth.orbit(12, 30.0, 10.0), 4946, 3286, 4627.3, 4649.5)
    files["syn_orbit"] = p
    p = os.path.join(out_dir, "syn_random.json")
    synth.write_cameras_json(p, synth.random_poses(16, seed=3), 1600, 1200, 1111.1, 1100.0)
    files["syn_random"] = p
    p = os.path.join(out_dir, "syn_portrait.json")
    poses = [(np.array([3.0, 1.5, -12.0 + i]), synth.look_at_c2w([3.0, 1.5, -12.0 + i], [0.5, 2.0 * i, 0.0]))
             for i in range(6)]
    synth.write_cameras_json(p, poses, 1080, 1920, 1700.0, 1650.0)
    files["syn_portrait"] = p
    return files


def run_harness(json_path: str, row, harness: str = HARNESS):
    w, h, fovy, near, far, override = row
    with tempfile.TemporaryDirectory(prefix="gps_cam_") as out:
        subprocess.run([harness, "camera", json_path, out, str(w), str(h), repr(fovy), repr(near), repr(far),
                        str(override)], check=True, capture_output=True, timeout=120)
        return np.load(os.path.join(out, "camera_matrices.npy")), np.load(os.path.join(out, "camera_resolution.npy"))


def main():
    if not os.path.exists(HARNESS):
        sys.exit("reference harness not built (oracle/ref/build_ref.sh)")
    fix = {"settings": np.array(SETTINGS, np.float64)}
    with tempfile.TemporaryDirectory(prefix="gps_camjson_") as d:
        files = synthetic_json_files(d)
        for name in sorted(glob.glob(os.path.join(REF_ROOT, "assets", "cameras", "*.json"))):
            stem = os.path.splitext(os.path.basename(name))[0].encode("ascii", "ignore").decode()
            files["asset_" + stem] = name
        for tag, path in sorted(files.items()):
            fix[f"{tag}__sha256"] = np.frombuffer(hashlib.sha256(open(path, "rb").read()).digest(), np.uint8)
            for i, row in enumerate(SETTINGS):
                mats, res = run_harness(path, row)
                fix[f"{tag}__{i}__mats"] = mats[:MAX_CAMERAS]
                fix[f"{tag}__{i}__res"] = res[:MAX_CAMERAS]
    out = os.path.join(HERE, "camera_ref.npz")
    np.savez_compressed(out, **fix)
    print("wrote", out, len(fix), "arrays")


if __name__ == "__main__":
    main()
