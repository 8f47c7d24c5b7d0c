"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, to check the
CUDA path against; the library never does.  Build with `make -C oracle` (done by __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_float, c_int, c_int32, c_uint32, c_uint64, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
LIB64_PATH = os.path.join(_HERE, "_build", "liboracle64.so")  # the same estimator in double precision
_libs = {}


def lib(fp64: bool = False):
    if fp64 not in _libs:
        path = LIB64_PATH if fp64 else LIB_PATH
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {_HERE}`")
        L = ctypes.CDLL(path)
        L.oracle_create.restype = c_void_p
        L.oracle_create.argtypes = [c_void_p, c_uint64, c_void_p, c_int]
        L.oracle_free.argtypes = [c_void_p]
        L.oracle_render_frame.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.oracle_splat_workload.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_uint32, c_uint32, c_int]
        L.oracle_preprocess.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]
        L.oracle_get_buffer.argtypes = [c_void_p, c_void_p]
        L.oracle_buffer_entries.restype = c_uint64
        L.oracle_buffer_entries.argtypes = [c_void_p]
        L.oracle_get_hiz.argtypes = [c_void_p, c_void_p]
        L.oracle_hiz_size.restype = c_uint64
        L.oracle_hiz_size.argtypes = [c_void_p]
        L.oracle_last_workload.argtypes = [c_void_p, c_void_p, POINTER(c_uint32), POINTER(c_uint32)]
        L.oracle_get_survivors.argtypes = [c_void_p, c_void_p, c_void_p]
        L.oracle_get_blocks.argtypes = [c_void_p, c_void_p, POINTER(c_uint32), POINTER(c_uint32)]
        L.oracle_kat.argtypes = [c_void_p] * 3 + [c_int] + [c_void_p] * 7
        L.oracle_splat_index.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]
        L.oracle_depth_key.argtypes = [c_void_p, c_int, c_float, c_float, c_void_p]
        L.oracle_rgb36.argtypes = [c_void_p, c_int, c_void_p]
        _libs[fp64] = L
    return _libs[fp64]


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


class Oracle:
    """One scene + settings + frame state, rendered on the CPU with `threads` threads."""

    def __init__(self, gaussians: np.ndarray, settings, threads: int = 1, fp64: bool = False):
        """fp64: the same estimator (same sample streams) in double precision."""
        self._lib = lib(fp64)
        g = np.ascontiguousarray(gaussians, dtype=np.float32)
        self._g = g
        self.settings = settings
        self.n = g.shape[0]
        self._h = self._lib.oracle_create(_p(g), g.shape[0], ctypes.addressof(settings), threads)

    def render(self, cam):
        s = self.settings
        img = np.zeros((s.height, s.width, 3), np.float32)
        dep = np.zeros((s.height, s.width), np.float32)
        self._lib.oracle_render_frame(self._h, ctypes.addressof(cam), _p(img), _p(dep))
        return img, dep

    def preprocess(self, cam, first_pass=True):
        counts = np.zeros(self.n, np.uint32)
        mask = np.zeros((self.n + 31) // 32, np.uint32)
        colors = np.zeros((self.n, 3), np.float32)
        self._lib.oracle_preprocess(self._h, ctypes.addressof(cam), int(first_pass), _p(counts), _p(mask), _p(colors))
        return counts, mask, colors

    def splat_workload(self, cam, frame_seed, surv_gid, surv_start, points, clear=True):
        g = np.ascontiguousarray(surv_gid, np.uint32)
        st = np.ascontiguousarray(surv_start, np.uint32)
        self._lib.oracle_splat_workload(self._h, ctypes.addressof(cam), frame_seed, _p(g), _p(st), g.size, points, int(clear))

    def buffer(self):
        out = np.zeros(self._lib.oracle_buffer_entries(self._h), np.uint64)
        self._lib.oracle_get_buffer(self._h, _p(out))
        return out

    def hiz(self):
        out = np.zeros(self._lib.oracle_hiz_size(self._h), np.float32)
        self._lib.oracle_get_hiz(self._h, _p(out))
        return out

    def workload(self):
        pp = np.zeros(2, np.uint32)
        sv = c_uint32()
        tot = c_uint32()
        self._lib.oracle_last_workload(self._h, _p(pp), byref(sv), byref(tot))
        gid = np.zeros(sv.value, np.uint32)
        start = np.zeros(sv.value, np.uint32)
        self._lib.oracle_get_survivors(self._h, _p(gid), _p(start))
        return {"points_pass": pp, "survivors": sv.value, "total": tot.value, "surv_gid": gid, "surv_start": start}

    def blocks(self):
        n = (self.n + 3) // 4 + 1
        nodes = np.zeros(n * 6, np.float32)
        pb = c_uint32()
        cnt = c_uint32()
        self._lib.oracle_get_blocks(self._h, _p(nodes), byref(pb), byref(cnt))
        return nodes[: cnt.value * 6].reshape(-1, 6), pb.value

    def close(self):
        if self._h:
            self._lib.oracle_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def settings_host(**overrides):
    """A gps_settings with the reference's defaults (render_settings.cuh:36-265), filled here so
    that the CPU baseline never loads the CUDA library; only the struct layout is shared."""
    import gpsplat  # the ctypes struct definitions only; the shared library is not loaded

    st = gpsplat.Settings()
    d = dict(width=1920, height=1080, supersampling_factor=2, samples_per_pixel=1, max_number_of_points=250_000_000,
             fovy=45.0, near_view_plane=0.2, far_view_plane=10000.0, enable_hierarchical_culling=1,
             fully_disable_hierarchical_culling=0, enable_occlusion_culling=1, occlusion_culling_min_reduce_count=0,
             cull_small_gaussians=0, use_unbiased_2d_splatting=1, reduce_point_count=1, accumulation_mode=0,
             sort_morton_order=0, immediate_splat_threshold=0, points_per_thread=0)
    d.update(overrides)
    for k, v in d.items():
        if k == "background":
            for i in range(3):
                st.background[i] = float(v[i])
        else:
            setattr(st, k, v)
    return st


def camera_host(position, c2w, settings, frame: int):
    """The viewer's per-frame camera (main.cu:141-157, camera.cpp:88-156) in numpy: view =
    diag(1,-1,-1,1) * inverse([R | p]) with R the camera-to-world rotation (columns right, down,
    forward), glm::perspective with NDC z in [-1, 1], normalised frustum planes of proj*view.
    Float64 arithmetic rounded to float32: the CPU baseline's cameras, not the parity path's."""
    import gpsplat

    R = np.asarray(c2w, np.float64)
    M = np.eye(4)
    M[:3, :3] = R
    M[:3, 3] = np.asarray(position, np.float64)
    view = np.diag([1.0, -1.0, -1.0, 1.0]) @ np.linalg.inv(M)
    f = 1.0 / np.tan(np.radians(settings.fovy) / 2.0)
    aspect = settings.width / settings.height
    n, fa = settings.near_view_plane, settings.far_view_plane
    proj = np.zeros((4, 4))
    proj[0, 0] = f / aspect
    proj[1, 1] = f
    proj[2, 2] = -(fa + n) / (fa - n)
    proj[2, 3] = -2.0 * fa * n / (fa - n)
    proj[3, 2] = -1.0
    vp = proj @ view
    planes = np.stack([vp[3] + vp[0], vp[3] - vp[0], vp[3] + vp[1], vp[3] - vp[1], vp[3] + vp[2], vp[3] - vp[2]])
    planes /= np.linalg.norm(planes[:, :3], axis=1, keepdims=True)
    cam = gpsplat.Camera()
    cam.view[:] = [float(x) for x in view.T.astype(np.float32).reshape(-1)]
    cam.proj[:] = [float(x) for x in proj.T.astype(np.float32).reshape(-1)]
    cam.position[:] = [float(x) for x in np.asarray(position, np.float32)]
    cam.frustum_planes[:] = [float(x) for x in planes.astype(np.float32).reshape(-1)]
    cam.frame = int(frame)
    cam.camera_moved = 1
    return cam


def kat(idx, frame, x):
    idx = np.ascontiguousarray(idx, np.uint32)
    frame = np.ascontiguousarray(frame, np.uint32)
    x = np.ascontiguousarray(x, np.float32)
    n = idx.size
    out = {
        "seed": np.zeros((n, 2), np.uint32),
        "pcg": np.zeros((n, 2), np.uint32),
        "pcgf": np.zeros((n, 2), np.float32),
        "dilog": np.zeros(n, np.float32),
        "invdilog": np.zeros(n, np.float32),
        "poisson": np.zeros(n, np.uint32),
        "sround": np.zeros(n, np.int32),
    }
    lib().oracle_kat(_p(idx), _p(frame), _p(x), n, _p(out["seed"]), _p(out["pcg"]), _p(out["pcgf"]), _p(out["dilog"]),
                     _p(out["invdilog"]), _p(out["poisson"]), _p(out["sround"]))
    return out


def splat_index(xs, ys, ps, npass, width):
    xs, ys, ps = (np.ascontiguousarray(v, np.int32) for v in (xs, ys, ps))
    out = np.zeros(xs.size, np.int64)
    lib().oracle_splat_index(_p(xs), _p(ys), _p(ps), xs.size, npass, width, _p(out))
    return out


def depth_key(d, near, far):
    d = np.ascontiguousarray(d, np.float32)
    out = np.zeros(d.size, np.uint64)
    lib().oracle_depth_key(_p(d), d.size, near, far, _p(out))
    return out


def rgb36(rgb):
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.zeros(rgb.shape[0], np.uint64)
    lib().oracle_rgb36(_p(rgb), rgb.shape[0], _p(out))
    return out


def morton_order(gaussians: np.ndarray) -> np.ndarray:
    """The --sort-morton-order permutation (gaussian_loader.cu:363-424): bounds of the means
    (glm::min/max fold from FLT_MAX / -FLT_MAX, lines 365-377; a NaN never wins its
    comparisons), rel = safe_div(mean - min, max - min) (lines 249-255, 387), 21-bit
    truncation of rel * (2^21 - 1) (line 388), morton3D21 interleave x -> bit 3b, y -> 3b+1,
    z -> 3b+2 (lines 257-265), then a stable sort of the keys (thrust::sort_by_key on uint64
    keys, a radix sort, lines 397-404).  order[j] = the input index of the j-th Gaussian."""
    g = np.asarray(gaussians, np.float32)
    n = g.shape[0]
    if n == 0:
        return np.zeros(0, np.uint32)
    mean = np.ascontiguousarray(g[:, 0:3], np.float32)
    nan = np.isnan(mean)
    fmax = np.float32(np.finfo(np.float32).max)
    mn = np.minimum(np.where(nan, fmax, mean).min(axis=0), fmax).astype(np.float32)
    mx = np.maximum(np.where(nan, -fmax, mean).max(axis=0), -fmax).astype(np.float32)
    den = (mx - mn).astype(np.float32)
    num = (mean - mn).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(den != 0, num / np.where(den != 0, den, np.float32(1)), np.float32(0)).astype(np.float32)
        scaled = (rel * np.float32((1 << 21) - 1)).astype(np.float32)
        q = np.where(np.isfinite(scaled), scaled, 0).astype(np.int64) & 0x1FFFFF
    key = np.zeros(n, np.uint64)
    for bit in range(21):
        for c in range(3):
            key |= ((q[:, c].astype(np.uint64) >> np.uint64(bit)) & np.uint64(1)) << np.uint64(3 * bit + c)
    return np.argsort(key, kind="stable").astype(np.uint32)
