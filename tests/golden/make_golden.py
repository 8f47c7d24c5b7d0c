"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own kernels.

Runs the headless reference build (oracle/_ref/<variant>/ref_harness, built from the
reference's sources by oracle/ref/build_ref.sh) on a B200 for small seeded scenes and camera
sequences, and stores what it produced:

  kat.npz          known answers of the reference's device helpers (seeds, PCG, dilog and its
                   inverse, Box-Muller, corrected Box-Muller, Poisson, stochastic rounding,
                   Morton addressing, depth keys, background packing)
  case_<name>.npz  per-frame splat buffer, image, depth, Hi-Z chain, survivor masks, point
                   offsets, point count and SH colours, plus the camera records and a hash of
                   the PLY bytes the scene was generated as

Usage (on a GPU box, from the repository root):  python tests/golden/make_golden.py [case ...]
(all fixtures, or only the named cases; GPS_GOLDEN_OUT redirects the output directory)
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "gaussian-point-splatting_b200"))

import gpsplat  # noqa: E402
import gpsutil  # noqa: E402
import synth  # noqa: E402


def _cube_pose(i=0):
    p = np.array([1.5 * i, 0.7 * i, -30.0 + 2.0 * i])
    return (p, synth.look_at_c2w(p, [0.0, 0.0, 0.0]))


# name: (scene maker, scene tag, settings overrides, poses, harness variant, scene format)
CASES = {
    "plain_cube8k": (lambda: synth.cube(8000, seed=21), "cube8k_s21",
                     dict(width=160, height=90, supersampling_factor=1, samples_per_pixel=1,
                          fully_disable_hierarchical_culling=1, enable_occlusion_culling=0),
                     [_cube_pose(0)], "fp32", gpsplat.GPS_SCENE_FP32),
    "ss2spp2_occl_cube8k": (lambda: synth.cube(8000, seed=21), "cube8k_s21",
                            dict(width=160, height=90, supersampling_factor=2, samples_per_pixel=2,
                                 fully_disable_hierarchical_culling=1, enable_occlusion_culling=1),
                            [_cube_pose(0), _cube_pose(1)], "fp32", gpsplat.GPS_SCENE_FP32),
    "town_cull_12k": (lambda: synth.town(12000, seed=9), "town12k_s9",
                      dict(width=160, height=90, supersampling_factor=2, samples_per_pixel=1),
                      synth.orbit(2, 30.0, 10.0), "fp32", gpsplat.GPS_SCENE_FP32),
    "biased_cullsmall_cube8k": (lambda: synth.cube(8000, seed=21), "cube8k_s21",
                                dict(width=160, height=90, supersampling_factor=1, samples_per_pixel=2,
                                     fully_disable_hierarchical_culling=1, enable_occlusion_culling=0,
                                     use_unbiased_2d_splatting=0, cull_small_gaussians=1, background=(0.1, 0.4, 0.9)),
                                [_cube_pose(0)], "fp32", gpsplat.GPS_SCENE_FP32),
    "compressed_town8k": (lambda: synth.town(8000, seed=9), "town8k_s9",
                          dict(width=160, height=90, supersampling_factor=1, samples_per_pixel=1,
                               fully_disable_hierarchical_culling=1, enable_occlusion_culling=0),
                          synth.orbit(1, 30.0, 10.0), "compressed", gpsplat.GPS_SCENE_COMPRESSED),
    # ENABLE_IMMEDIATE_SPLATTING build: small Gaussians splatted inside the preprocess
    "immediate_occl_town12k": (lambda: synth.town(12000, seed=9), "town12k_s9",
                               dict(width=160, height=90, supersampling_factor=2, samples_per_pixel=2,
                                    immediate_splat_threshold=8),
                               synth.orbit(2, 30.0, 10.0), "immediate", gpsplat.GPS_SCENE_FP32),
    "immediate_biased_cube8k": (lambda: synth.cube(8000, seed=21), "cube8k_s21",
                                dict(width=160, height=90, supersampling_factor=2, samples_per_pixel=1,
                                     fully_disable_hierarchical_culling=1, enable_occlusion_culling=0,
                                     use_unbiased_2d_splatting=0, immediate_splat_threshold=4),
                                [_cube_pose(0)], "immediate", gpsplat.GPS_SCENE_FP32),
}
OUT = os.environ.get("GPS_GOLDEN_OUT", HERE)


def file_sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def make_kat(out_path):
    exe = gpsutil.ref_harness("fp32")
    d = tempfile.mkdtemp()
    subprocess.run([exe, "kat", d], check=True)
    arrays = {os.path.splitext(f)[0]: np.load(os.path.join(d, f)) for f in os.listdir(d) if f.endswith(".npy")}
    np.savez_compressed(out_path, **arrays)


def make_case(name):
    make, tag, overrides, poses, variant, fmt = CASES[name]
    ply = gpsutil.cached_ply(tag, make)
    s = gpsplat.default_settings(**overrides)
    cams = gpsutil.cameras_for(s, poses)
    frames, extra = gpsutil.run_reference(ply, s, cams, variant=variant)
    out = {"ply_sha256": np.array(file_sha256(ply)), "frames": np.array(len(frames))}
    rec = np.zeros(len(cams), gpsutil.CAM_DTYPE)
    for i, c in enumerate(cams):
        dd = gpsplat.camera_to_numpy(c)
        for k in ("view", "proj", "position"):
            rec[i][k] = dd[k]
        rec[i]["planes"] = dd["planes"]
        rec[i]["frame"] = c.frame
        rec[i]["camera_moved"] = c.camera_moved
    out["cameras"] = rec
    n = None
    for i, fr in enumerate(frames):
        n = fr["colors"].shape[0]
        ml = gpsutil.mask_bits(fr["mask_last"], n)
        mo = gpsutil.mask_bits(fr["mask_other"], n)
        valid = ml | mo if overrides.get("enable_occlusion_culling", 1) else ml
        out[f"f{i}_buffer"] = fr["buffer"]
        out[f"f{i}_checksum"] = fr["buffer_checksum"]
        out[f"f{i}_image"] = fr["image"]
        out[f"f{i}_depth"] = fr["depth"]
        out[f"f{i}_hiz"] = fr["hiz"]
        out[f"f{i}_mask_last"] = fr["mask_last"]
        out[f"f{i}_mask_other"] = fr["mask_other"]
        out[f"f{i}_offsets"] = fr["offsets"]
        out[f"f{i}_stats"] = fr["stats"]
        out[f"f{i}_color_ids"] = np.nonzero(valid)[0].astype(np.uint32)
        out[f"f{i}_colors"] = fr["colors"][valid]
        out[f"f{i}_derived"] = fr["derived"]
        if "culled" in fr:
            out[f"f{i}_culled"] = fr["culled"]
    for k, v in extra.items():
        out[k] = v
    np.savez_compressed(os.path.join(OUT, f"case_{name}.npz"), **out)


def main():
    if gpsutil.ref_harness("fp32") is None:
        raise SystemExit("reference harness not built: run oracle/ref/build_ref.sh where the reference sources are")
    names = sys.argv[1:] or list(CASES)
    if not sys.argv[1:]:
        make_kat(os.path.join(OUT, "kat.npz"))
    for name in names:
        make_case(name)
        print("wrote", name, flush=True)


if __name__ == "__main__":
    main()
