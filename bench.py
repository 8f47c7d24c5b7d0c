#!/usr/bin/env python3
"""Headline benchmark: Gaussians/s (and ms/frame) of the point-splatting frame path at
1080p, 4 spp, on the synthetic 16M-Gaussian town (supersampling 2, K = 4 points per thread,
BVH-block + Hi-Z occlusion culling, TAA), stepping a 120-frame orbit one keyframe per frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference] [--workload town16m|cube1m]

One step = one frame (render + TAA post-process) through the library's C-ABI frame loop.
`value` is whole-job Gaussians/s = N_scene x frames / device time (max over ranks); `e2e`
repeats the timed loop through the same public call with the per-frame camera handed over
from host memory and the u8 frame read back into pinned host memory every step.

--gpus N > 1 (under torchrun): N independent replicas (the reference renders one view on one
GPU; the path has no cross-GPU exchange), each rank on its own orbit phase; weak scaling.
--impl reference: the reference has no CPU implementation of the path, so the CPU restatement
of its algorithm (oracle/) is timed on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gaussian-point-splatting_b200"))

import synth  # noqa: E402

SCENE_CACHE = os.path.join("/tmp", "gps_b200_scenes")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_spec(name: str):
    if name == "town16m":
        return dict(n=16_000_000, kind="town", width=1920, height=1080, ss=2, spp=4, reduce=1, hier=1, occl=1,
                    taa=1, frames=120)
    if name == "town4m":  # profiling-size variant of the headline workload
        return dict(n=4_000_000, kind="town", width=1920, height=1080, ss=2, spp=4, reduce=1, hier=1, occl=1,
                    taa=1, frames=120)
    if name == "town256m":  # the town tiled 4 x 4 in the half-precision format
        return dict(n=16_000_000, tiles=4, kind="town", fmt="half", width=1920, height=1080, ss=2, spp=4, reduce=1,
                    hier=1, occl=1, taa=1, frames=120)
    if name == "town4m_tiled":  # profiling-size variant of town256m: the 4M town tiled 2 x 2 (16M)
        return dict(n=4_000_000, tiles=2, kind="town", fmt="half", width=1920, height=1080, ss=2, spp=4, reduce=1,
                    hier=1, occl=1, taa=1, frames=120)
    if name == "cube1m":
        return dict(n=1_000_000, kind="cube", width=640, height=360, ss=1, spp=1, reduce=1, hier=0, occl=0, taa=0,
                    frames=1)
    raise SystemExit(f"unknown workload {name}")


def load_scene_host(spec) -> np.ndarray:
    """Activated CPUGaussian array (N x 59 float32), cached on local disk per box."""
    return load_scene_files(spec)[1]


def load_scene_files(spec):
    """(PLY path, activated host array) of the workload's scene, generated once per box.  The
    PLY (3DGS binary layout, with the bvh_sorted_order comment) is what the library's
    gps_scene_load_ply and the reference's own loader read; the activated array feeds the CPU
    baseline."""
    os.makedirs(SCENE_CACHE, exist_ok=True)
    stem = os.path.join(SCENE_CACHE, f"{spec['kind']}{spec['n']}")
    ply, act = stem + ".ply", stem + "_act.npy"
    if os.path.exists(ply) and os.path.exists(act):
        return ply, np.load(act, mmap_mode="r")
    t = time.time()
    raw = synth.town(spec["n"]) if spec["kind"] == "town" else synth.cube(spec["n"])
    if not os.path.exists(ply):
        tmp = ply + f".{os.getpid()}.tmp"
        raw.write_ply(tmp)
        os.replace(tmp, ply)
    g = synth.activate(raw)
    del raw
    log(f"generated {spec['kind']} scene with {spec['n']} Gaussians in {time.time() - t:.1f}s")
    tmp = act + f".{os.getpid()}.tmp.npy"
    np.save(tmp, g)
    os.replace(tmp, act)
    return ply, g


def poses_for(spec):
    if spec["kind"] == "town":
        return synth.orbit(spec["frames"], 30.0, 10.0)
    p = np.array([0.0, 0.0, -30.0])
    return [(p, synth.look_at_c2w(p, [0.0, 0.0, 0.0]))]


def settings_for(gpsplat, spec):
    return gpsplat.default_settings(
        width=spec["width"], height=spec["height"], supersampling_factor=spec["ss"], samples_per_pixel=spec["spp"],
        reduce_point_count=spec["reduce"], enable_hierarchical_culling=spec["hier"],
        fully_disable_hierarchical_culling=0 if spec["hier"] else 1, enable_occlusion_culling=spec["occl"],
        accumulation_mode=gpsplat.GPS_ACCUM_TAA if spec["taa"] else gpsplat.GPS_ACCUM_NONE)


def make_cameras(gpsplat, settings, poses, count, phase):
    cams = []
    for i in range(count):
        p, r = poses[(phase + i) % len(poses)]
        c = gpsplat.camera_from_pose(p, np.asarray(r, np.float32).T, settings, i + 1)
        c.camera_moved = 1
        cams.append(c)
    return cams


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max clock, throttle reasons)."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend: str = "nccl"):
    """Replica plumbing: one process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from torchrun)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def orbit_phase(rank: int, world: int, frames: int) -> int:
    """First orbit keyframe of a replica: the ranks start evenly spread around the orbit."""
    return (rank * frames) // max(1, world)


def max_over_ranks(x: float, world: int) -> float:
    """Device time of the job = the slowest replica's (all ranks take part, in the same order)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------------
# CPU baseline (the oracle, oracle/oracle.cpp) on a bounded sample of the workload
# ---------------------------------------------------------------------------------
# bytes the preprocess reads per Gaussian it loads (opacity + geometry) and per survivor (SH),
# by scene format: FP32 SoA (16 B position+opacity, 16 B rotation, 16 B scale; 192 B SH),
# the reference's compressed format (16 B quantised geometry + 1 B opacity; 64 B compact SH),
# and the half format (16 B + 16 B records; 48 B int8 AC coefficients)
PREPROCESS_BYTES = {"fp32": (48.0, 192.0), "compressed": (17.0, 64.0), "half": (32.0, 48.0)}


def stage_rooflines(stages, spec, st, entries, passes, w, h, peak):
    """Achieved algorithmic GB/s of the HBM-bound stages, per launch, against the measured copy
    peak.  Algorithmic bytes per launch (counts from the device counters of the last frame):
      preprocess  per Gaussian whose attributes were read (device tally, after the block cull
                  and pass 2's previous-mask test): its geometry; per survivor: its SH, the
                  64-byte splat record and the 4-byte count; per 32 Gaussians read: the mask
                  word read and written
      scan        per 32 Gaussians: the mask word, read twice; per survivor: its count read
                  twice and 8 bytes of workload written
      resolve     8 per splat-buffer entry + 16 per pixel (final) / 4 (depth-only), averaged
      clear       8 per splat-buffer entry"""
    out = {}
    n = spec["n"] * spec.get("tiles", 1) ** 2
    read = (st.gaussians_read_one + st.gaussians_read_two) / max(1, passes)
    surv = (st.survivors_one + st.survivors_two) / max(1, passes)
    geom, sh = PREPROCESS_BYTES[spec.get("fmt", "fp32")]
    model = {
        "preprocess": read * geom + surv * (sh + 64.0 + 4.0) + read / 32.0 * 8.0 if read > 0 else None,
        "scan": n / 4.0 + surv * (8.0 + 8.0),
        "resolve": 8.0 * entries + (10.0 if passes == 2 else 16.0) * w * h,
        "clear": 8.0 * entries,
    }
    for k, b in model.items():
        ms, launches = stages.get(k, (0.0, 0))
        if b is None or ms <= 0 or launches <= 0:
            continue
        if k == "scan":
            launches = max(1, launches // 2)  # two launches per pass: tile scan, downsweep
        per = ms / launches
        gbs = b / (per / 1000.0) / 1e9
        out[k] = {"achieved_gbs": gbs, "frac": gbs / peak, "ms_per_launch": per, "algorithmic_bytes": b}
        if k == "preprocess":
            out[k]["gaussians_read_per_pass"] = read
            out[k]["survivors_per_pass"] = surv
    return out


def profile_figure(kernel: str, workload: str, key: str):
    """A per-launch figure of the dominant kernel from the committed ncu summary of the same
    workload (profiles/<kernel>_traffic_<workload>.md, `key: value` lines, averaged over a
    frame's launches): traffic_per_launch_bytes = dram__bytes_read.sum + dram__bytes_write.sum,
    atomics_per_launch = l1tex__t_sectors_pipe_lsu_mem_global_op_red.sum.  None when absent."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_traffic_{workload}.md")
    try:
        with open(path) as f:
            for ln in f:
                if ln.startswith(key + ":"):
                    return float(ln.split(":")[1]), os.path.relpath(path, ROOT)
    except OSError:
        pass
    return None, None


def measured_traffic(kernel: str, spec, workload: str):
    return profile_figure(kernel, workload, "traffic_per_launch_bytes")


def atomic_peaks(gpsplat, entries: int, stream):
    """Measured rate of 64-bit atomicMin on random slots (gps_measure_atomic_min_rate): over a
    buffer the size of the splat buffer, and over one that fits in L2."""
    import ctypes

    import torch

    lib = gpsplat.load_library()
    out = {}
    for name, words in (("splat_buffer", entries), ("l2_resident", 8 << 20)):
        buf = torch.empty(int(words), dtype=torch.int64, device="cuda")
        rate = ctypes.c_double(0.0)
        st = lib.gps_measure_atomic_min_rate(ctypes.c_void_p(buf.data_ptr()), int(words), 5, ctypes.byref(rate),
                                             ctypes.c_void_p(stream.cuda_stream))
        out[name] = {"atomics_per_s": rate.value if st == 0 else None, "buffer_bytes": int(words) * 8}
        del buf
    return out


def host_cameras(spec, settings, poses, count, phase=0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return [oracle.camera_host(*poses[(phase + i) % len(poses)], settings, i + 1) for i in range(count)]


def host_settings(spec):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle.settings_host(
        width=spec["width"], height=spec["height"], supersampling_factor=spec["ss"], samples_per_pixel=spec["spp"],
        reduce_point_count=spec["reduce"], enable_hierarchical_culling=spec["hier"],
        fully_disable_hierarchical_culling=0 if spec["hier"] else 1, enable_occlusion_culling=spec["occl"],
        accumulation_mode=1 if spec["taa"] else 2)


def cpu_frames(g_host, spec, frames: int, threads: int, budget_s: float = 1e9):
    """Full frames of the workload (the whole scene, its camera path from the first keyframe)
    rendered by the CPU oracle with `threads` host threads; returns (frames done, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    s = host_settings(spec)
    cams = host_cameras(spec, s, poses_for(spec), frames)
    o = oracle.Oracle(np.ascontiguousarray(g_host), s, threads=threads)
    t0 = time.time()
    done = 0
    for c in cams:
        o.render(c)
        done += 1
        if time.time() - t0 > budget_s:
            break
    dt = time.time() - t0
    o.close()
    return done, dt


def cpu_baseline(g_host, spec, frames_all: int = 2, frames_one: int = 1):
    """The CPU restatement of the estimator (oracle/) on the whole scene: `frames_all` frames on
    every host core, then `frames_one` frame(s) on one core."""
    cores = os.cpu_count() or 1
    n = g_host.shape[0]
    f_all, dt_all = cpu_frames(g_host, spec, frames_all, cores)
    out = {"value": n * f_all / dt_all, "unit": "Gaussians/s", "cores": cores, "kind": "port",
           "sample": f"the whole {n}-Gaussian scene, {f_all} frames of its camera path from the first keyframe, "
                     f"{dt_all:.1f}s on {cores} threads"}
    if frames_one > 0:
        f_one, dt_one = cpu_frames(g_host, spec, frames_one, 1)
        out["one_thread"] = {"value": n * f_one / dt_one, "unit": "Gaussians/s", "cores": 1,
                             "sample": f"the whole scene, {f_one} frame(s), {dt_one:.1f}s"}
    return out


def run_reference_arm(args, spec, world, rank):
    """The reference has no CPU implementation of this path; its CPU restatement (oracle/) is
    timed on every host core, whole frames of the same scene and camera path: one warm-up frame,
    then up to `steps` frames within a bounded time.  Nothing here loads the CUDA library."""
    if rank != 0:
        return 0
    g = load_scene_host(spec)
    cores = os.cpu_count() or 1
    warm, _ = cpu_frames(g, spec, args.warmup, cores, budget_s=30.0)  # page the scene in
    done, dt = cpu_frames(g, spec, args.steps, cores, budget_s=REFERENCE_ARM_BUDGET_S)
    value = spec["n"] * done / dt
    cb = {"value": value, "unit": "Gaussians/s", "cores": cores, "kind": "port",
          "sample": f"the whole {spec['n']}-Gaussian scene, {done} of {args.steps} frames of its camera path "
                    f"({dt:.1f}s; frames stop after {REFERENCE_ARM_BUDGET_S:.0f}s), {warm} warm-up frame(s)"}
    line = {"impl": "reference", "metric": "Gaussians/sec", "value": value, "unit": "Gaussians/s", "n_gpus": world,
            "steps": done, "warmup": warm, "ms_per_step": 1000.0 * dt / max(1, done), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {spec['kind']}, see synth.py)",
            "config": {"workload": args.workload, "gaussians": spec["n"], "resolution": [spec["width"], spec["height"]],
                       "supersampling": spec["ss"], "spp": spec["spp"], "culling": bool(spec["hier"]),
                       "taa": bool(spec["taa"])},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "Gaussians/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


REFERENCE_ARM_BUDGET_S = 150.0


def reference_cuda(gpsplat, ply, spec, settings, cams, warmup, mine_ms):
    """Frame time of the reference's own CUDA kernels on this GPU, same PLY, cameras and
    settings: the headless build of the reference's sources (oracle/ref/build_ref.sh; its
    GaussianPointSplatting::render plus the RenderServer post-process, timed per frame with CUDA
    events, its per-pass host synchronisations included), in its FP32 and its default
    compressed format.  `mine_ms` maps each format to this library's ms/frame on the same frames."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import tempfile

    import gpsutil

    out = {}
    work = tempfile.mkdtemp(prefix="gps_refcuda_")
    camf = os.path.join(work, "cams.bin")
    gpsutil.write_camera_file(camf, cams)
    for variant in ("fp32", "compressed"):
        exe = gpsutil.ref_harness(variant)
        if exe is None:
            out[variant] = {"unavailable": "reference build missing (oracle/ref/build_ref.sh)"}
            continue
        args = [exe, "render", ply, work, camf] + gpsutil.harness_args(settings, taa_race_free=False) + \
            ["--checksum-only", "--time", "--warmup", str(warmup), "--dump-frames", "0", "--no-post-dump"]
        t = time.time()
        res = subprocess.run(args, capture_output=True, text=True, timeout=1800)
        if res.returncode != 0:
            out[variant] = {"unavailable": f"reference harness failed ({res.returncode}): {res.stderr[-300:]}"}
            continue
        ref = json.loads([ln for ln in res.stdout.splitlines() if ln.startswith("{")][-1])
        entry = {"reference_ms_per_frame": ref["ms_per_frame"], "frames": ref["frames"], "wall_s": time.time() - t}
        ready = [ln for ln in res.stderr.splitlines() if ln.startswith("reference scene ready in")]
        if ready:  # the reference's PLY load + scene upload + BVH build (its GaussianPointSplatting constructor)
            entry["reference_scene_load_s"] = float(ready[-1].split()[4])
        if mine_ms.get(variant):
            entry["ms_per_frame"] = mine_ms[variant]
            entry["speedup"] = ref["ms_per_frame"] / mine_ms[variant]
        out[variant] = entry
    return out


def ingest(gpsplat, ply, g_host, load_ply_s):
    """The load path around the frame path: PLY parse, the scene build through the PLY loader,
    and the --sort-morton-order reorder (gaussian_loader.cu:363-424) on the host (the
    reference's host keys + sort) and on the device (keys, stable radix sort and gather in HBM),
    on the workload's own Gaussians in a shuffled order."""
    import torch

    n = g_host.shape[0]
    out = {"gaussians": n, "load_ply_s": load_ply_s}
    t = time.perf_counter()
    gpsplat.ply_read(ply)
    out["ply_parse_s"] = time.perf_counter() - t
    perm = np.random.default_rng(0x5EED).permutation(n)
    shuffled = np.ascontiguousarray(g_host[perm])
    t = time.perf_counter()
    host_order = gpsplat.morton_order(shuffled, on_device=False)
    out["morton_order_host_s"] = time.perf_counter() - t
    gpsplat.morton_order(shuffled[: 1 << 16], on_device=True)  # first-use costs outside the timing
    t = time.perf_counter()
    dev_order = gpsplat.morton_order(shuffled, on_device=True)
    out["morton_order_device_s"] = time.perf_counter() - t
    out["orders_equal"] = bool(np.array_equal(host_order, dev_order))
    del host_order, dev_order
    for mode, key in ((1, "scene_build_host_reorder_s"), (2, "scene_build_device_reorder_s")):
        torch.cuda.synchronize()
        t = time.perf_counter()
        sc = gpsplat.Scene.from_host_sorted(shuffled, gpsplat.GPS_SCENE_FP32, mode)
        torch.cuda.synchronize()
        out[key] = time.perf_counter() - t
        sc.close()
    t = time.perf_counter()
    sc = gpsplat.Scene.from_host(shuffled, gpsplat.GPS_SCENE_FP32, presorted=False)
    torch.cuda.synchronize()
    out["scene_build_no_reorder_s"] = time.perf_counter() - t
    sc.close()
    return out


def time_frames(gpsplat, scene, settings, cams, warmup, stream):
    """Device ms per frame of the frame loop over `cams` after `warmup` of them."""
    import torch

    r = gpsplat.Renderer(scene, settings)
    loop = gpsplat.FrameLoop(r)
    for c in cams[:warmup]:
        loop.step(c, stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for c in cams[warmup:]:
        loop.step(c, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    loop.close()
    r.close()
    return e0.elapsed_time(e1) / max(1, len(cams) - warmup)


# ---------------------------------------------------------------------------------
# batched multi-view workload: 64 views of the 16M town, views/s batch vs plain
# ---------------------------------------------------------------------------------
BATCH_RES = [(320, 180), (640, 360), (1280, 720), (1920, 1080)]
BATCH_SPP = [1, 2, 4, 8, 16]


def run_batch_workload(args, world, rank, local):
    """One step = one batch of 64 views (seeded random poses inside the town, resolution and
    spp drawn from BATCH_RES x BATCH_SPP, supersampling 2, BVH + Hi-Z culling) rendered by
    gps_batch_render; the same 64 views rendered one at a time through gps_renderer_reset +
    gps_render_frame (one renderer per view configuration, one stream) is the plain path timed
    beside it, and the two must agree bit for bit."""
    import torch

    torch.cuda.set_device(local)
    import gpsplat

    gpsplat.load_library()
    spec = workload_spec("town16m")
    g_host = load_scene_host(spec)
    scene = gpsplat.Scene.from_host(np.ascontiguousarray(g_host), presorted=True)
    base = dict(supersampling_factor=2, enable_hierarchical_culling=1, enable_occlusion_culling=1)
    rng = np.random.default_rng(64 + rank)
    poses = synth.random_poses(64, seed=7 + rank)
    views = []
    for i, (p, r) in enumerate(poses):
        w, h = BATCH_RES[int(rng.integers(len(BATCH_RES)))]
        spp = BATCH_SPP[int(rng.integers(len(BATCH_SPP)))]
        s = gpsplat.default_settings(**base, width=w, height=h, samples_per_pixel=spp)
        cam = gpsplat.camera_from_pose(p, np.asarray(r, np.float32).T, s, i + 1)
        views.append(dict(cam=cam, w=w, h=h, spp=spp, s=s, img=torch.empty((h, w, 3), device="cuda"),
                          dep=torch.empty((h, w), device="cuda"), pimg=torch.empty((h, w, 3), device="cuda"),
                          pdep=torch.empty((h, w), device="cuda")))
    arr = gpsplat.Batch.views([(v["cam"], v["w"], v["h"], v["spp"], v["img"].data_ptr(), v["dep"].data_ptr()) for v in views])
    cap = gpsplat.default_settings(**base, width=1920, height=1080, samples_per_pixel=16)
    batch = gpsplat.Batch(scene, cap, 1920, 1080, 16, workers=8)
    batch.use_graph(True)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    # the autotuner over K in {1, 2, 4, 8} x workers, each K's best kept for the record
    search = {}
    for k in (1, 2, 4, 8):
        batch.set_points_per_thread(k)
        w_k, ms_k = batch.autotune(arr, rounds=1, stream=sh)
        search[k] = {"workers": w_k, "ms_per_batch": ms_k}
    chosen_k = min(search, key=lambda k: search[k]["ms_per_batch"])
    chosen, tune_ms = search[chosen_k]["workers"], search[chosen_k]["ms_per_batch"]
    batch.set_points_per_thread(chosen_k)
    batch.workers = chosen
    renderers = {}  # the plain path: the reference's K (ss^2 points per thread)
    for v in views:
        key = (v["w"], v["h"], v["spp"])
        if key not in renderers:
            renderers[key] = gpsplat.Renderer(scene, v["s"])

    def plain_round():
        for v in views:  # each view as a fresh single-view render, like the batch's
            r = renderers[(v["w"], v["h"], v["spp"])]
            r.reset(sh)
            r.render(v["cam"], v["pimg"].data_ptr(), v["pdep"].data_ptr(), sh)

    # bit-exactness: every batch view against a plain render with the batch's (tuned) K
    batch.render(arr, sh)
    torch.cuda.synchronize()
    same = True
    for v in views:
        sk = gpsplat.default_settings(**base, width=v["w"], height=v["h"], samples_per_pixel=v["spp"],
                                      points_per_thread=chosen_k)
        rk = gpsplat.Renderer(scene, sk)
        rk.render(v["cam"], v["pimg"].data_ptr(), v["pdep"].data_ptr(), sh)
        torch.cuda.synchronize()
        same = same and torch.equal(v["img"].view(torch.int32), v["pimg"].view(torch.int32)) and \
            torch.equal(v["dep"].view(torch.int32), v["pdep"].view(torch.int32))
        rk.close()
    for _ in range(args.warmup):
        batch.render(arr, sh)
        plain_round()
    torch.cuda.synchronize()

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    batch_ms = timed(lambda: batch.render(arr, sh))
    clocks = sampler.stop()
    plain_ms = timed(plain_round)
    # end to end: every view's image read back to pinned host memory each step
    host = [torch.empty((v["h"], v["w"], 3), dtype=torch.float32, pin_memory=True) for v in views]

    def e2e_step():
        batch.render(arr, sh)
        for v, hb in zip(views, host):
            hb.copy_(v["img"], non_blocking=True)

    with torch.cuda.stream(stream):
        e2e_ms = timed(e2e_step)
    d2h = sum(v["w"] * v["h"] * 12 for v in views)
    n_views = len(views) * args.steps * world
    value = n_views / (batch_ms / 1000.0)
    line = {
        "metric": "views/sec", "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": batch_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded town and poses, see synth.py)",
        "config": {"workload": "batch64", "gaussians": scene.count, "views_per_step": len(views),
                   "resolutions": BATCH_RES, "spp": BATCH_SPP, "supersampling": 2, "culling": True,
                   "l2": "inputs larger than L2 (scene 3.8 GB)", "parallelism": f"replicas x{world}"},
        "plain": {"value": n_views / (plain_ms / 1000.0), "unit": "views/s", "ms_per_step": plain_ms / args.steps},
        "speedup_vs_plain": plain_ms / batch_ms,
        "bit_exact_vs_plain_same_k": bool(same),
        "autotune": {"workers": chosen, "points_per_thread": chosen_k, "ms_per_batch": tune_ms,
                     "per_k": {str(k): v for k, v in search.items()}, "workers_searched": [1, 2, 4, 8]},
        "graph": dict(zip(("instantiations", "updates"), batch.graph_stats())),
        "clocks": clocks,
        "e2e": {"value": n_views / (e2e_ms / 1000.0), "unit": "views/s", "h2d_bytes_per_step": len(bytes(arr)),
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / args.steps},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    for r in renderers.values():
        r.close()
    scene.close()
    return 0


# ---------------------------------------------------------------------------------
# serving workload: Poisson arrivals over the 16M FP32 and 256M half-precision towns
# ---------------------------------------------------------------------------------
SERVE_RES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]
SERVE_SPP = [1, 4, 16]
SERVE_RATES = [50.0, 200.0, 1000.0]


def run_serve_workload(args, world, rank, local):
    """Requests arrive as a Poisson process (SERVE_RATES req/s, `--steps` x 20 requests per
    rate): 70% for the 16M town (FP32), 30% for the 256M town (half precision, 4 x 4 tiles),
    seeded poses, resolution from SERVE_RES, spp from SERVE_SPP, supersampling 2, culling on.
    The server (4 workers, continuous admission) is measured beside the plain loop (one worker,
    one request at a time, same arrivals): served views/s and p50/p99 latency from submission
    to the end of the request's GPU work."""
    import torch

    torch.cuda.set_device(local)
    import gpsplat

    gpsplat.load_library()
    g_host = load_scene_host(workload_spec("town16m"))
    town = gpsplat.Scene.from_host(np.ascontiguousarray(g_host), presorted=True)
    half = gpsplat.Scene.from_host(np.ascontiguousarray(g_host), gpsplat.GPS_SCENE_HALF, presorted=True)
    ext = synth.TOWN_EXTENT
    big = half.tile([[(i - 1.5) * ext, (j - 1.5) * ext] for j in range(4) for i in range(4)])
    half.close()
    scenes = [town, big]
    base = dict(supersampling_factor=2, enable_hierarchical_culling=1, enable_occlusion_culling=1)
    n_req = max(20, args.steps * 20)
    rng = np.random.default_rng(5 + rank)
    poses = synth.random_poses(n_req, seed=21 + rank)
    reqs = []
    for i in range(n_req):
        w, h = SERVE_RES[int(rng.integers(len(SERVE_RES)))]
        spp = SERVE_SPP[int(rng.integers(len(SERVE_SPP)))]
        s = gpsplat.default_settings(**base, width=w, height=h, samples_per_pixel=spp)
        p, r = poses[i]
        cam = gpsplat.camera_from_pose(p, np.asarray(r, np.float32).T, s, i + 1)
        reqs.append((i, 0 if rng.random() < 0.7 else 1, cam, w, h, spp))
    cap = gpsplat.default_settings(**base, width=3840, height=2160, samples_per_pixel=16)

    def run(server, rate, seed):
        gaps = np.random.default_rng(seed).exponential(1.0 / rate, size=len(reqs))
        t0 = time.perf_counter()
        due = t0
        for q, gap in zip(reqs, gaps):
            due += gap
            delay = due - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            server.submit(*q)
        server.drain(1200.0)
        wall = time.perf_counter() - t0
        done = server.poll(len(reqs) + 8)
        assert len(done) == len(reqs) and all(c[1] == 0 for c in done), "a request failed"
        lat = np.array([c[4] for c in done])
        return {"rate_req_s": rate, "views_per_s": len(reqs) / wall, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "workers_used": len({c[2] for c in done})}

    results = {}
    for mode, workers, budget in (("server", 4, None), ("server_unlimited", 4, 0), ("plain", 1, None)):
        server = gpsplat.Server(scenes, cap, 3840, 2160, 16, workers=workers)
        if budget is not None:
            server.set_admission(budget)
        for q in reqs[: min(8, len(reqs))]:  # warm-up
            server.submit(*q)
        server.drain(1200.0)
        server.poll(64)
        results[mode] = [run(server, rate, 100 + k) for k, rate in enumerate(SERVE_RATES)]
        server.close()
    top = results["server"][-1]
    line = {
        "metric": "served views/sec", "value": top["views_per_s"] * world, "unit": "views/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / top["views_per_s"] * 20,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (16M town), f16/int8 storage (256M town)",
        "data": "synthetic (seeded towns, poses and Poisson arrivals, see synth.py)",
        "config": {"workload": "serve", "requests_per_rate": len(reqs), "scenes": {"town16m_fp32": 0.7, "town256m_half": 0.3},
                   "resolutions": SERVE_RES, "spp": SERVE_SPP, "supersampling": 2, "rates_req_s": SERVE_RATES,
                   "server_workers": 4, "parallelism": f"replicas x{world}"},
        "server": results["server"], "server_no_admission_budget": results["server_unlimited"], "plain": results["plain"],
        "speedup_vs_plain_at_top_rate": top["views_per_s"] / results["plain"][-1]["views_per_s"],
        "e2e": {"value": top["views_per_s"] * world, "unit": "views/s", "h2d_bytes_per_step": 20 * 128,
                "d2h_bytes_per_step": 0, "note": "requests handed over from host memory; images stay on the device"},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for sc in scenes:
        sc.close()
    return 0


# ---------------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="town16m", choices=["town16m", "town4m", "town256m", "town4m_tiled", "cube1m", "batch64", "serve"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true", help="skip timing the reference's CUDA build")
    ap.add_argument("--quick-cpu", action="store_true", help="CPU baseline on all cores only (no 1-thread frame)")
    ap.add_argument("--no-ingest", action="store_true", help="skip timing the PLY parse and the Morton reorder")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_init()
    if args.workload == "batch64":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference renders one view per call; the "
                                  "batch64 views/s comparison is against this library's plain single-view path"}))
            return 0
        return run_batch_workload(args, world, rank, local)
    if args.workload == "serve":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no request server; the "
                                  "serve comparison is against this library's one-request-at-a-time loop"}))
            return 0
        return run_serve_workload(args, world, rank, local)
    spec = workload_spec(args.workload)
    if args.impl == "reference":
        return run_reference_arm(args, spec, world, rank)

    import torch

    torch.cuda.set_device(local)
    import gpsplat

    gpsplat.load_library()
    ply, g_host = load_scene_files(spec)
    t = time.time()
    if spec.get("fmt") == "half":
        base_scene = gpsplat.Scene.from_host(np.ascontiguousarray(g_host), gpsplat.GPS_SCENE_HALF, presorted=True)
        k = spec["tiles"]
        ext = synth.TOWN_EXTENT
        scene = base_scene.tile([[(i - (k - 1) / 2) * ext, (j - (k - 1) / 2) * ext] for j in range(k) for i in range(k)])
        base_scene.close()
    else:
        # through the reference-facing loader (gps_scene_load_ply), as a drop-in user loads it
        scene = gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_FP32)
    load_ply_s = time.time() - t
    log(f"rank {rank}: scene uploaded in {load_ply_s:.1f}s")
    s = settings_for(gpsplat, spec)
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    poses = poses_for(spec)
    phase = orbit_phase(rank, world, len(poses))
    total = args.warmup + args.steps
    cams = make_cameras(gpsplat, s, poses, total, phase)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    # warm-up
    for c in cams[: args.warmup]:
        loop.step(c, sh)
    torch.cuda.synchronize()
    r.enable_timing(False)

    # ---- device-timed region: K frames, inputs resident (splat buffer 2x L2 every frame) ----
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for c in cams[args.warmup:]:
        loop.step(c, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    dev_ms = e0.elapsed_time(e1)
    dev_ms_max = max_over_ranks(dev_ms, world)
    st = r.stats()
    launches_per_frame = st.kernel_launches

    # ---- per-stage times (separate timed pass with CUDA events between stages) ----
    r.enable_timing(True)
    r.stage_times(reset=True)
    for c in cams[args.warmup:]:
        loop.step(c, sh)
    torch.cuda.synchronize()
    stages = r.stage_times(reset=True)
    r.enable_timing(False)

    # ---- end to end through the public call with host buffers ----
    h, w = s.height, s.width
    host_frames = [torch.empty((h, w, 3), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    cam_bytes = len(bytes(cams[0]))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for i, c in enumerate(cams[args.warmup:]):
        loop.step(c, sh)  # camera handed over from host memory
        loop.read_async(host_frames[i % 2].numpy(), sh)  # u8 frame back to pinned host memory,
    loop.read_wait()                                       # overlapping the next frame's render
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)
    wall_e2e = time.perf_counter() - t0
    barrier(world)

    n_scene = scene.count
    K = args.steps
    value = n_scene * K * world / (dev_ms_max / 1000.0)
    e2e_value = n_scene * K * world / (e2e_ms / 1000.0)

    # roofline of the dominant kernel
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launches = stages[dom]
    per_launch_ms = dom_ms / max(1, dom_launches)
    entries = r.splat_buffer()[1]
    surv = st.survivors_one + st.survivors_two
    passes = 2 if spec["occl"] else 1
    if dom == "splat":
        # compulsory traffic of a splat launch: each survivor's 64-byte record and 8 bytes of
        # workload, one read and one write of every splat-buffer entry
        alg_bytes = (72.0 * surv / passes) + 16.0 * entries
    elif dom == "resolve":
        alg_bytes = 8.0 * entries + 16.0 * w * h
    else:
        alg_bytes = stage_rooflines(stages, spec, st, entries, passes, w, h, hbm_peak).get(dom, {}).get(
            "algorithmic_bytes", 8.0 * entries)
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic, traffic_src = measured_traffic(dom, spec, args.workload)
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": per_launch_ms,
                "traffic_source": traffic_src}

    # the splat's own bound: 64-bit atomicMin on random slots of its buffer
    splat_atomic = None
    if "splat" in stages:
        peaks_atomic = atomic_peaks(gpsplat, entries, stream)
        reds, reds_src = profile_figure("splat", args.workload, "atomics_per_launch")
        s_ms, s_launches = stages["splat"]
        per = s_ms / max(1, s_launches)
        peak_rate = peaks_atomic["splat_buffer"]["atomics_per_s"]
        splat_atomic = {"bound": "l2_atomic_min_u64", "peak": peak_rate, "peak_l2_resident": peaks_atomic["l2_resident"]["atomics_per_s"],
                        "unit": "atomics/s", "ms_per_launch": per, "atomics_per_launch": reds, "atomics_source": reds_src,
                        "achieved": (reds / (per / 1000.0)) if reds else None}
        if reds and peak_rate:
            splat_atomic["frac"] = splat_atomic["achieved"] / peak_rate

    l2_note = (f"inputs larger than L2: the {8 * entries / 1e6:.0f} MB splat buffer is cleared, scattered into and "
               f"resolved every frame; the preprocess reads the attributes of the Gaussians that pass the block cull "
               f"({(st.gaussians_read_one + st.gaussians_read_two) / passes / 1e6:.1f}M per pass)")
    line = {
        "metric": "Gaussians/sec", "value": value, "unit": "Gaussians/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": dev_ms_max / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {spec['kind']}, see synth.py)",
        "config": {"workload": args.workload, "gaussians": n_scene, "resolution": [w, h], "supersampling": spec["ss"],
                   "spp": spec["spp"], "points_per_thread": spec["ss"] ** 2 if spec["reduce"] else 1,
                   "culling": bool(spec["hier"]), "occlusion": bool(spec["occl"]), "taa": bool(spec["taa"]),
                   "camera_path": f"{len(poses)}-frame orbit r=30 h=10" if spec["kind"] == "town" else "static",
                   "l2": l2_note, "parallelism": f"replicas x{world}"},
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "Gaussians/s", "h2d_bytes_per_step": cam_bytes,
                "d2h_bytes_per_step": h * w * 3, "ms_per_step": e2e_ms / K, "wall_s": wall_e2e},
        "gpu_launches": int(launches_per_frame * K),
        "roofline": roofline,
        "splat_atomic_roofline": splat_atomic,
        "stages_ms_per_frame": {k: v[0] / K for k, v in stages.items()},
        "stage_rooflines": stage_rooflines(stages, spec, st, entries, passes, w, h, hbm_peak),
        "points_per_frame": [st.num_points_one, st.num_points_two],
        "survivors_per_frame": [st.survivors_one, st.survivors_two],
        "gaussians_read_per_frame": [st.gaussians_read_one, st.gaussians_read_two],
        "screen_order_per_pass": [st.screen_order_one, st.screen_order_two],
    }
    if spec.get("fmt") == "half":
        line["dtype"] = "f16/int8 storage, f32 arithmetic"
        line["config"]["format"] = "half (GPS_SCENE_HALF), town tiled %dx%d" % (spec["tiles"], spec["tiles"])
    loop.close()
    r.close()
    if rank == 0 and world == 1 and spec.get("fmt") != "half" and not args.no_reference_cuda:
        # the reference's own CUDA kernels on the same PLY, cameras and settings, beside this
        # library's frame loop on the same frames in the same two formats
        mine = {"fp32": time_frames(gpsplat, scene, s, cams, args.warmup, stream)}
        comp = gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_COMPRESSED)
        mine["compressed"] = time_frames(gpsplat, comp, s, cams, args.warmup, stream)
        comp.close()
        line["reference_cuda"] = reference_cuda(gpsplat, ply, spec, s, cams, args.warmup, mine)
    if rank == 0 and world == 1 and spec.get("fmt") != "half" and not args.no_ingest:
        line["ingest"] = ingest(gpsplat, ply, g_host, load_ply_s)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if spec.get("fmt") == "half":
            line["cpu_baseline"] = {"value": None, "unit": "Gaussians/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": "none: the CPU restatement has no half-precision format and the tiled "
                                              "256M scene does not fit its host-memory layout"}
        else:
            line["cpu_baseline"] = cpu_baseline(g_host, spec, frames_all=2, frames_one=0 if args.quick_cpu else 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
