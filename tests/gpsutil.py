"""Helpers shared by the tests: library loading, device<->host copies, camera files for the
reference harness, running the harness and this library on identical inputs.

The reference harness (oracle/_ref/<variant>/ref_harness, built from the reference's own
sources by oracle/ref/build_ref.sh) is a checker only; nothing here is on the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gaussian-point-splatting_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

import gpsplat  # noqa: E402
import synth  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")

_cudart = None


def cudart():
    global _cudart
    if _cudart is None:
        import torch  # noqa: F401  (loads the CUDA runtime that ships with torch)

        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                _cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if _cudart is None:
            raise OSError("libcudart not found")
        _cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        _cudart.cudaMemcpy.restype = ctypes.c_int
        _cudart.cudaDeviceSynchronize.restype = ctypes.c_int
    return _cudart


def d2h(ptr: int, count: int, dtype) -> np.ndarray:
    """Copies `count` elements of `dtype` from a raw device pointer to a new numpy array."""
    out = np.empty(count, dtype=dtype)
    if count:
        rc = cudart().cudaMemcpy(out.ctypes.data, ctypes.c_void_p(ptr), out.nbytes, 2)
        assert rc == 0, f"cudaMemcpy failed ({rc})"
    return out


def sync():
    assert cudart().cudaDeviceSynchronize() == 0


def ref_harness(variant: str = "fp32") -> str | None:
    p = os.path.join(REF_DIR, variant, "ref_harness")
    return p if os.path.exists(p) else None


CAM_DTYPE = np.dtype([("view", "<f4", 16), ("proj", "<f4", 16), ("position", "<f4", 3), ("planes", "<f4", 24),
                      ("frame", "<i4"), ("camera_moved", "<i4")])


def cameras_for(settings, poses, first_frame: int = 1, moved=None):
    cams = []
    for i, (p, r) in enumerate(poses):
        basis_cols = np.asarray(r, np.float32).T  # rows of this array = basis columns
        cam = gpsplat.camera_from_pose(p, basis_cols, settings, first_frame + i)
        cam.camera_moved = 1 if (moved is None or moved) else 0
        cams.append(cam)
    return cams


def write_camera_file(path: str, cams):
    rec = np.zeros(len(cams), CAM_DTYPE)
    for i, c in enumerate(cams):
        d = gpsplat.camera_to_numpy(c)
        rec[i]["view"] = d["view"]
        rec[i]["proj"] = d["proj"]
        rec[i]["position"] = d["position"]
        rec[i]["planes"] = d["planes"]
        rec[i]["frame"] = c.frame
        rec[i]["camera_moved"] = c.camera_moved
    rec.tofile(path)


def harness_args(s, taa_race_free: bool = True) -> list[str]:
    a = ["--res", str(s.width), str(s.height), "--ss", str(s.supersampling_factor), "--spp", str(s.samples_per_pixel),
         "--max-points", str(s.max_number_of_points), "--near", repr(float(s.near_view_plane)), "--far",
         repr(float(s.far_view_plane)), "--fovy", repr(float(s.fovy))]
    if not s.reduce_point_count:
        a.append("--one-point-per-thread")
    if not s.enable_hierarchical_culling:
        a.append("--disable-hierarchical-culling")
    if s.fully_disable_hierarchical_culling:
        a.append("--fully-disable-hierarchical-culling")
    if not s.enable_occlusion_culling:
        a.append("--disable-occlusion-culling")
    if s.cull_small_gaussians:
        a.append("--cull-small")
    if not s.use_unbiased_2d_splatting:
        a.append("--biased")
    if s.occlusion_culling_min_reduce_count:
        a += ["--min-reduce", str(s.occlusion_culling_min_reduce_count)]
    if any(s.background[i] != 0 for i in range(3)):
        a += ["--background"] + [repr(float(s.background[i])) for i in range(3)]
    if s.immediate_splat_threshold > 0:
        a += ["--immediate-threshold", str(s.immediate_splat_threshold)]
    if s.sort_morton_order:
        a.append("--sort-morton-order")
    if s.accumulation_mode == gpsplat.GPS_ACCUM_TAA:
        # the harness runs the reference's own temporalRender so that no pixel reads a
        # neighbour's blended value (its in-place blend otherwise races; see ref_harness.cu);
        # timing runs keep the reference's own single launch
        a.append("--taa-race-free" if taa_race_free else "--taa")
    elif s.accumulation_mode == gpsplat.GPS_ACCUM_NONE:
        a.append("--no-accumulation")
    return a


def run_reference(ply: str, settings, cams, variant="fp32", checksum_only=False, timeout=900):
    """Runs the reference's kernels (headless harness) and returns per-frame dumps."""
    exe = ref_harness(variant)
    if exe is None:
        raise FileNotFoundError("reference harness not built")
    out = tempfile.mkdtemp(prefix="gps_ref_")
    camf = os.path.join(out, "cams.bin")
    write_camera_file(camf, cams)
    args = [exe, "render", ply, out, camf] + harness_args(settings)
    if checksum_only:
        args.append("--checksum-only")
    res = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"reference harness failed ({res.returncode}): {res.stderr[-2000:]}")
    frames = []
    for i in range(len(cams)):
        d = {}
        for name in ("derived", "buffer_checksum", "buffer", "image", "image_pre_post", "depth", "post_u8", "hiz",
                     "offsets", "mask_last",
                     "mask_other", "indices", "colors", "stats", "culled"):
            p = os.path.join(out, f"f{i:03d}_{name}.npy")
            if os.path.exists(p):
                d[name] = np.load(p)
        frames.append(d)
    extra = {}
    for name in ("bvh_nodes", "bvh_gpb") + (("scene_cpu",) if settings.sort_morton_order else ()):
        p = os.path.join(out, f"{name}.npy")
        if os.path.exists(p):
            extra[name] = np.load(p)
    return frames, extra


def run_mine(scene, settings, cams, full=True):
    """Renders `cams` through the library's frame loop; returns per-frame arrays shaped like
    the reference harness dumps."""
    r = gpsplat.Renderer(scene, settings)
    loop = gpsplat.FrameLoop(r)
    w, h = settings.width, settings.height
    frames = []
    n = scene.count
    for cam in cams:
        loop.step(cam)
        sync()
        st = r.stats()
        d = {"stats_obj": st}
        d["derived"] = r.derived(cam)
        bptr, entries = r.splat_buffer()
        buf = d2h(bptr, entries, np.uint64)
        d["buffer_checksum"] = gpsplat.buffer_checksum(buf)
        if full:
            d["buffer"] = buf
        a = cam.frame % 2
        _, col_a, _ = loop.buffers(a)
        u8, _, dep_b = loop.buffers(1 - a)
        d["image"] = d2h(col_a, w * h * 3, np.float32).reshape(h, w, 3)
        if settings.accumulation_mode == gpsplat.GPS_ACCUM_TAA:
            _, pre, _ = loop.buffers(2)
            d["image_pre_post"] = d2h(pre, w * h * 3, np.float32).reshape(h, w, 3)
        else:
            d["image_pre_post"] = d["image"]
        d["depth"] = d2h(dep_b, w * h, np.float32).reshape(h, w)
        d["post_u8"] = d2h(u8, w * h * 3, np.uint8).reshape(h, w, 3)
        v = r.debug_view()
        d["hiz"] = d2h(v.hiz, v.hiz_size, np.float32)
        words = (n + 31) // 32
        d["mask_last"] = d2h(v.mask_last, words, np.uint32)
        d["mask_other"] = d2h(v.mask_other, words, np.uint32)
        counts = d2h(v.counts, n, np.uint32)
        d["counts"] = counts
        d["surv_gid"] = d2h(v.surv_gid, v.survivors, np.uint32)
        d["surv_start"] = d2h(v.surv_start, v.survivors, np.uint32)
        d["points"] = int(v.points)
        if full:
            rec = d2h(v.records, n * 16, np.float32).reshape(n, 16)
            d["colors_rec"] = rec[:, 9:12]
        if v.block_words:
            d["culled"] = d2h(v.block_culled, v.block_words, np.uint32)
            d["block_nodes"] = d2h(v.block_nodes, v.block_count * 8, np.float32).reshape(-1, 8)
            d["per_block"] = v.per_block
        frames.append(d)
    loop.close()
    r.close()
    return frames


def mask_bits(words: np.ndarray, n: int) -> np.ndarray:
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:n]
    return bits.astype(bool)


def written_mask(m: dict, n: int) -> np.ndarray:
    """The survivor mask the frame's last pass wrote.  The reference advances its mask pair only
    after a pass with points (workload_distributor.cu:107-111,145), so that is mask_last (its
    "previous" mask) after a pass with points and mask_other (its "current" one) after an
    empty pass; its weights array holds the exclusive scan over that mask either way."""
    return mask_bits(m["mask_last"] if m["points"] > 0 else m["mask_other"], n)


def offsets_from(counts: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Exclusive u32 scan of masked counts (what the reference leaves in its weights array)."""
    c = np.where(mask, counts, 0).astype(np.uint64)
    ex = np.concatenate([[0], np.cumsum(c)[:-1]]).astype(np.uint64)
    return (ex & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def indices_from(surv_gid: np.ndarray, counts_of_surv: np.ndarray, points: int) -> np.ndarray:
    return np.repeat(surv_gid, counts_of_surv)[:points].astype(np.uint32)


def cached_ply(name: str, make) -> str:
    """Writes a synthetic scene PLY once per process into a temp dir."""
    d = os.path.join(tempfile.gettempdir(), "gps_b200_scenes")
    os.makedirs(d, exist_ok=True)
    p = os.path.join(d, name + ".ply")
    if not os.path.exists(p):
        raw = make()
        tmp = p + ".tmp"
        raw.write_ply(tmp)
        os.replace(tmp, p)
    return p


def decode_png(data: bytes):
    """A minimal PNG reader for 8-bit RGB, filter type 0 (what gps_write_png writes)."""
    import struct
    import zlib

    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, ihdr, types = 8, b"", None, []
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(kind + body) == crc, kind
        types.append(kind)
        if kind == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    assert types[0] == b"IHDR" and types[-1] == b"IEND"
    w, h, depth, colour, _, _, interlace = ihdr
    assert (depth, colour, interlace) == (8, 2, 0)
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert (raw[:, 0] == 0).all()
    return raw[:, 1:].reshape(h, w, 3)

