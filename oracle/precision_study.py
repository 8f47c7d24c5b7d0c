#!/usr/bin/env python3
"""Image error of the GPU paths against the FP64 oracle (test infrastructure).

The FP64 oracle (oracle/_build/liboracle64.so) runs the same estimator with the same integer
sample streams in double precision. Each path is averaged over F frames with the same seeds
(frame indices 1..F), and each mean is compared with the FP64 oracle's mean:

* the GPU FP32 path: arithmetic error only;
* the GPU half-precision path (GPS_SCENE_HALF): format plus arithmetic error.

The oracle also runs once more with other seeds, which gives the sampling-noise level for
scale. Prints one JSON line: PSNR and max per-pixel error of each path vs FP64.

    python oracle/precision_study.py [--n 60000] [--frames 32] [--width 320 --height 180 --spp 4]
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gaussian-point-splatting_b200"))

import gpsplat  # noqa: E402
import gpsutil  # noqa: E402
import oracle  # noqa: E402
import synth  # noqa: E402


def psnr(a, b):
    return float(10.0 * np.log10(1.0 / max(np.mean((a - b) ** 2), 1e-20)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=60000)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--width", type=int, default=320)
    ap.add_argument("--height", type=int, default=180)
    ap.add_argument("--spp", type=int, default=4)
    args = ap.parse_args()
    import torch

    raw = synth.town(args.n, seed=5)
    g = synth.activate(raw)
    s = gpsplat.default_settings(width=args.width, height=args.height, samples_per_pixel=args.spp,
                                 max_number_of_points=8_000_000)
    pose = synth.orbit(8, 30.0, 10.0)[3]
    W, H, F = args.width, args.height, args.frames

    def cams(first):
        return [gpsutil.cameras_for(s, [pose], first_frame=first + f)[0] for f in range(F)]

    def gpu_mean(fmt, first):
        scene = gpsplat.Scene.from_host(g, fmt, presorted=True)
        r = gpsplat.Renderer(scene, s)
        img = torch.empty((H, W, 3), device="cuda")
        dep = torch.empty((H, W), device="cuda")
        tot = np.zeros((H, W, 3))
        for cam in cams(first):
            r.reset(0)
            r.render(cam, img.data_ptr(), dep.data_ptr(), 0)
            torch.cuda.synchronize()
            tot += img.cpu().numpy()
        r.close()
        scene.close()
        return np.clip(tot / F, 0, 1)

    def oracle_mean(first):
        tot = np.zeros((H, W, 3))
        for cam in cams(first):
            o = oracle.Oracle(g, s, threads=os.cpu_count() or 1, fp64=True)  # fresh: first frame each
            img, _ = o.render(cam)
            o.close()
            tot += img
        return np.clip(tot / F, 0, 1)

    ref = oracle_mean(1)
    other = oracle_mean(10001)
    fp32 = gpu_mean(gpsplat.GPS_SCENE_FP32, 1)
    half = gpu_mean(gpsplat.GPS_SCENE_HALF, 1)
    out = {"scene": f"town {args.n}", "view": [W, H], "spp": args.spp, "supersampling": 2, "frames": F,
           "fp32_vs_fp64": {"psnr_db": psnr(fp32, ref), "max_abs": float(np.abs(fp32 - ref).max())},
           "half_vs_fp64": {"psnr_db": psnr(half, ref), "max_abs": float(np.abs(half - ref).max())},
           "sampling_noise_fp64_other_seeds": {"psnr_db": psnr(other, ref), "max_abs": float(np.abs(other - ref).max())}}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
