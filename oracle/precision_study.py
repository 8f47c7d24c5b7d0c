#!/usr/bin/env python3
"""Image error of the GPU paths against the FP64 oracle (test infrastructure).

The FP64 oracle (oracle/_build/liboracle64.so) runs the same estimator with the same integer
sample streams in double precision. Each path is averaged over F frames with the same seeds
(frame indices 1..F), and each mean is compared with the FP64 oracle's mean:

* the GPU FP32 path: arithmetic error only;
* the GPU half-precision path (GPS_SCENE_HALF): format plus arithmetic error.

The oracle also runs once more with other seeds, which gives the sampling-noise level for
scale. Prints one JSON line per configuration: PSNR and max per-pixel error of each path vs
FP64 (`small`: the 60k town at 320x180; `c1`, `c2`, `c3`: the frame configurations at their
own resolution, c3 as a one-tile crop of the tiled town).

    python oracle/precision_study.py [--configs small,c1,c2,c3] [--frames 32] [--threads T]
    python oracle/precision_study.py --half-budget --frames 64   # CPU only
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


CONFIGS = {
    # name: (scene kind, Gaussians, width, height, supersampling, spp, culling, formats)
    "small": ("town", 60000, 320, 180, 2, 4, True, ("fp32", "half")),
    # the three frame configurations at their own resolution; c3 is a one-tile crop (16M) of
    # the 4 x 4 tiled 256M town, whose copies share one encoding up to their origins
    "c1": ("cube", 1_000_000, 640, 360, 1, 1, False, ("fp32",)),
    "c2": ("town", 16_000_000, 1920, 1080, 2, 4, True, ("fp32",)),
    "c3": ("town", 16_000_000, 1920, 1080, 2, 4, True, ("half",)),
}
FORMATS = {"fp32": gpsplat.GPS_SCENE_FP32, "half": gpsplat.GPS_SCENE_HALF}


# ---- GPS_SCENE_HALF's rounding, restated on the host (for the format's error budget) ----------
def _bf16_up(x):
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((b >> 16) + ((b & 0xFFFF) != 0)).astype(np.uint32) << 16).view(np.float32)


def half_emulated(g, positions="fixed16", ac="int8_band"):
    """The activated scene as the half format stores it: positions as 16-bit fixed-point (or, for
    comparison, FP16) offsets from 16-Gaussian block origins; FP16 opacity, scale, rotation and
    SH DC; AC terms as int8 on a bf16 per-band scale (or FP8 e4m3 on one per-Gaussian scale)."""
    import torch

    r = np.array(g, np.float32, copy=True)
    for b in range(0, r.shape[0], 16):
        p = r[b:b + 16, 0:3]
        lo, hi = p.min(axis=0), p.max(axis=0)
        o = (np.float32(0.5) * (lo + hi)).astype(np.float32)
        if positions == "fp16":
            r[b:b + 16, 0:3] = o + (p - o).astype(np.float16).astype(np.float32)
            continue
        k = np.float32(np.max(np.maximum(hi - o, o - lo)) / np.float32(32767))
        r[b:b + 16, 0:3] = o + (np.clip(np.rint((p - o) / k), -32767, 32767) * k if k > 0 else 0)
    r[:, 3:6] = r[:, 3:6].astype(np.float16).astype(np.float32)
    r[:, 51:59] = r[:, 51:59].astype(np.float16).astype(np.float32)
    a = r[:, 6:51]  # the 45 AC terms (sh[3:48] of the CPUGaussian layout)
    if ac == "fp8":
        m = np.abs(a).max(axis=1)
        k = np.where(m > 0, m / np.float32(448), 1).astype(np.float32)
        r[:, 6:51] = torch.from_numpy(a / k[:, None]).to(torch.float8_e4m3fn).to(torch.float32).numpy() * k[:, None]
    else:
        for lo_, hi_ in ((0, 9), (9, 24), (24, 45)):
            m = np.abs(a[:, lo_:hi_]).max(axis=1)
            k = _bf16_up(m / np.float32(127))
            with np.errstate(divide="ignore", invalid="ignore"):
                q = np.where(k[:, None] > 0, np.clip(np.rint(a[:, lo_:hi_] / k[:, None]), -127, 127), 0)
            r[:, 6 + lo_:6 + hi_] = q * k[:, None]
    return r


def half_budget(frames, threads, views=(3, 0, 5)):
    """Converged-image gap of the emulated half format to FP32 on the CPU oracle (FP32 build):
    64-frame means against a 512-frame FP32 mean of the 60k town at 320x180, ss 2, 4 spp, as
    the GPU test measures it, for the current format and for FP16 offsets / FP8 AC terms."""
    g = synth.activate(synth.town(60000, seed=5))
    s = gpsplat.default_settings(width=320, height=180, samples_per_pixel=4, max_number_of_points=4_000_000)
    variants = {"current": half_emulated(g), "fp16_offsets": half_emulated(g, positions="fp16"),
                "fp16_offsets_fp8_ac": half_emulated(g, positions="fp16", ac="fp8")}
    for view in views:
        pose = synth.orbit(8, 30.0, 10.0)[view]

        def mean(gg, first, count):
            tot = 0
            for f in range(count):
                cam = gpsutil.cameras_for(s, [pose], first_frame=first + f)[0]
                o = oracle.Oracle(gg, s, threads=threads)
                img, _ = o.render(cam)
                o.close()
                tot = tot + img
            return np.clip(tot / count, 0, 1)

        ref = mean(g, 1000, 512)
        a = mean(g, 1, frames)
        out = {"view": view, "frames": frames, "fp32_vs_ref_db": psnr(a, ref)}
        for name, q in variants.items():
            out[name + "_gap_db"] = psnr(a, ref) - psnr(mean(q, 1, frames), ref)
        print(json.dumps(out), flush=True)


def study(name, frames, threads, scenes):
    import torch

    kind, n, W, H, ss, spp, cull, formats = CONFIGS[name]
    key = (kind, n)
    if key not in scenes:
        scenes[key] = synth.activate(synth.town(n, seed=5) if kind == "town" else synth.cube(n))
    g = scenes[key]
    s = gpsplat.default_settings(width=W, height=H, supersampling_factor=ss, samples_per_pixel=spp,
                                 **({"max_number_of_points": 8_000_000} if name == "small" else {}),
                                 enable_hierarchical_culling=int(cull), fully_disable_hierarchical_culling=int(not cull),
                                 enable_occlusion_culling=int(cull))
    if kind == "town":
        pose = synth.orbit(8, 30.0, 10.0)[3]
    else:
        p = np.array([0.0, 0.0, -30.0])
        pose = (p, synth.look_at_c2w(p, [0.0, 0.0, 0.0]))

    def cams(first):
        return [gpsutil.cameras_for(s, [pose], first_frame=first + f)[0] for f in range(frames)]

    def gpu_mean(fmt, first):
        scene = gpsplat.Scene.from_host(g, FORMATS[fmt], presorted=True)
        r = gpsplat.Renderer(scene, s)
        img = torch.empty((H, W, 3), device="cuda")
        dep = torch.empty((H, W), device="cuda")
        tot = np.zeros((H, W, 3))
        for cam in cams(first):
            r.reset(0)  # every frame a first frame, as the oracle's
            r.render(cam, img.data_ptr(), dep.data_ptr(), 0)
            torch.cuda.synchronize()
            tot += img.cpu().numpy()
        r.close()
        scene.close()
        return np.clip(tot / frames, 0, 1)

    def oracle_mean(first):
        tot = np.zeros((H, W, 3))
        for cam in cams(first):
            o = oracle.Oracle(g, s, threads=threads, fp64=True)  # fresh: first frame each
            img, _ = o.render(cam)
            o.close()
            tot += img
        return np.clip(tot / frames, 0, 1)

    ref = oracle_mean(1)
    other = oracle_mean(10001)
    out = {"config": name, "scene": f"{kind} {n}", "view": [W, H], "supersampling": ss, "spp": spp,
           "culling": cull, "frames": frames,
           "sampling_noise_fp64_other_seeds": {"psnr_db": psnr(other, ref), "max_abs": float(np.abs(other - ref).max())}}
    for fmt in formats:
        m = gpu_mean(fmt, 1)
        out[f"{fmt}_vs_fp64"] = {"psnr_db": psnr(m, ref), "max_abs": float(np.abs(m - ref).max())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="small", help="comma-separated: " + ",".join(CONFIGS))
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--half-budget", action="store_true", help="the half format's gap, emulated on the CPU oracle")
    args = ap.parse_args()
    if args.half_budget:
        half_budget(args.frames, args.threads)
        return
    scenes = {}
    for name in args.configs.split(","):
        print(json.dumps(study(name, args.frames, args.threads, scenes)), flush=True)


if __name__ == "__main__":
    main()
