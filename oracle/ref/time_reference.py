#!/usr/bin/env python3
"""Frame time of the reference's own CUDA kernels beside this library's, same scene, cameras
and settings, on one GPU.

The reference path is the headless harness built from the reference's sources by
build_ref.sh (oracle/_ref/<variant>/ref_harness): GaussianPointSplatting::render plus the
RenderServer post-process per frame, timed with CUDA events around each frame (its per-pass
host synchronisations included, as in the reference).  This library's path is the frame loop
(gps_frame_loop_step) timed the same way.  Test infrastructure: it measures the reference, it
is not part of the product.

    python oracle/ref/time_reference.py [--n 16000000] [--frames 30] [--warmup 3] [--variant fp32|compressed]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "gaussian-point-splatting_b200"))

import gpsplat  # noqa: E402
import gpsutil  # noqa: E402
import synth  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=16_000_000)
    ap.add_argument("--frames", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--variant", default="fp32", choices=["fp32", "compressed"])
    ap.add_argument("--workload", default="town", choices=["town", "cube"],
                    help="town: 1080p ss 2, 4 spp, culling, TAA, orbit; cube: 640x360 ss 1, 1 spp, no culling, static camera")
    args = ap.parse_args()
    import torch

    exe = gpsutil.ref_harness(args.variant)
    if exe is None:
        raise SystemExit("reference harness not built (oracle/ref/build_ref.sh)")
    work = tempfile.mkdtemp(prefix="gps_time_ref_")
    ply = os.path.join(work, f"{args.workload}{args.n}.ply")
    t = time.time()
    (synth.town(args.n) if args.workload == "town" else synth.cube(args.n)).write_ply(ply)
    print(f"scene written in {time.time() - t:.1f}s", file=sys.stderr)
    total = args.warmup + args.frames
    if args.workload == "town":
        s = gpsplat.default_settings(width=1920, height=1080, supersampling_factor=2, samples_per_pixel=4,
                                     accumulation_mode=gpsplat.GPS_ACCUM_TAA)
        cams = gpsutil.cameras_for(s, synth.orbit(120, 30.0, 10.0)[:total])
    else:
        s = gpsplat.default_settings(width=640, height=360, supersampling_factor=1, samples_per_pixel=1,
                                     fully_disable_hierarchical_culling=1, enable_occlusion_culling=0,
                                     accumulation_mode=gpsplat.GPS_ACCUM_NONE)
        p = np.array([0.0, 0.0, -30.0])
        cams = gpsutil.cameras_for(s, [(p, synth.look_at_c2w(p, [0.0, 0.0, 0.0]))] * total)
    camf = os.path.join(work, "cams.bin")
    gpsutil.write_camera_file(camf, cams)
    res = subprocess.run([exe, "render", ply, work, camf] + gpsutil.harness_args(s, taa_race_free=False) +
                         ["--checksum-only", "--time", "--warmup", str(args.warmup), "--dump-frames", "0",
                          "--no-post-dump"], capture_output=True, text=True, timeout=3000)
    if res.returncode != 0:
        raise SystemExit(res.stderr[-2000:])
    ref = json.loads([ln for ln in res.stdout.splitlines() if ln.startswith("{")][-1])

    fmt = gpsplat.GPS_SCENE_FP32 if args.variant == "fp32" else gpsplat.GPS_SCENE_COMPRESSED
    scene = gpsplat.Scene.from_ply(ply, fmt)
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    for c in cams[: args.warmup]:
        loop.step(c)
    torch.cuda.synchronize()
    ms = []
    for c in cams[args.warmup:]:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        loop.step(c)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    out = {"workload": args.workload, "gaussians": args.n, "format": args.variant, "frames": args.frames,
           "resolution": [s.width, s.height], "supersampling": s.supersampling_factor, "spp": s.samples_per_pixel,
           "culling": bool(s.enable_occlusion_culling), "taa": s.accumulation_mode == gpsplat.GPS_ACCUM_TAA,
           "reference_ms_per_frame": ref["ms_per_frame"], "this_ms_per_frame": float(np.mean(ms)),
           "speedup": ref["ms_per_frame"] / float(np.mean(ms))}
    print(json.dumps(out))
    loop.close()
    r.close()
    scene.close()


if __name__ == "__main__":
    main()
