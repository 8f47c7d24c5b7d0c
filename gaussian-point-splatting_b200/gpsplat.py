"""ctypes binding of libgps_b200.so, the B200-native Gaussian point-splatting frame path.

The Python side is a thin mirror of the C-ABI in include/gps_b200.h, which in turn mirrors
the reference's render-pass interface (RenderPass::render, src/core/rendering/render_pass.cuh:17-24;
GaussianPointSplatting, src/core/rendering/passes/gaussian_point_splatting.cu:599-816) and its
settings (RenderSettings, src/render_settings.cuh:36-103).  There is no CPU fallback: loading
fails loudly when the shared library is missing, and every call raises GpsError on a non-zero
status.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_char, c_char_p, c_float, c_int32, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# GPS_B200_LIBRARY points at a libgps_b200.so built elsewhere (e.g. with other tuning options)
LIB_PATH = os.environ.get("GPS_B200_LIBRARY") or os.path.join(_HERE, "libgps_b200.so")

GPS_SCENE_FP32 = 0
GPS_SCENE_COMPRESSED = 1
GPS_SCENE_HALF = 2
GPS_ACCUM_PROGRESSIVE = 0
GPS_ACCUM_TAA = 1
GPS_ACCUM_NONE = 2

STATUS_NAMES = {
    0: "GPS_OK",
    1: "GPS_ERR_INVALID_ARGUMENT",
    2: "GPS_ERR_IO",
    3: "GPS_ERR_FORMAT",
    4: "GPS_ERR_CUDA",
    5: "GPS_ERR_OUT_OF_MEMORY",
    6: "GPS_ERR_SIZE",
    7: "GPS_ERR_DEVICE_TIMEOUT",
}

# CPUGaussian layout (gaussian_types.cuh:89-100): mean[3], sh[48], opacity, scale[3], rotation[4]
GAUSSIAN_FLOATS = 59
OFF_MEAN, OFF_SH, OFF_OPACITY, OFF_SCALE, OFF_ROT = 0, 3, 51, 52, 55


class GpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Settings(ctypes.Structure):
    _fields_ = [
        ("width", c_int32),
        ("height", c_int32),
        ("supersampling_factor", c_int32),
        ("samples_per_pixel", c_int32),
        ("max_number_of_points", c_int32),
        ("fovy", c_float),
        ("near_view_plane", c_float),
        ("far_view_plane", c_float),
        ("enable_hierarchical_culling", c_int32),
        ("fully_disable_hierarchical_culling", c_int32),
        ("enable_occlusion_culling", c_int32),
        ("occlusion_culling_min_reduce_count", c_int32),
        ("cull_small_gaussians", c_int32),
        ("use_unbiased_2d_splatting", c_int32),
        ("reduce_point_count", c_int32),
        ("background", c_float * 3),
        ("accumulation_mode", c_int32),
        ("sort_morton_order", c_int32),
        ("immediate_splat_threshold", c_int32),
        ("points_per_thread", c_int32),
    ]


class Camera(ctypes.Structure):
    _fields_ = [
        ("view", c_float * 16),
        ("proj", c_float * 16),
        ("position", c_float * 3),
        ("frustum_planes", c_float * 24),
        ("frame", c_int32),
        ("camera_moved", c_int32),
    ]


class View(ctypes.Structure):
    """gps_view: one view of a batch."""
    _fields_ = [("camera", Camera), ("width", c_int32), ("height", c_int32), ("samples_per_pixel", c_int32),
                ("d_image", c_void_p), ("d_depth", c_void_p)]


class Request(ctypes.Structure):
    """gps_request: one render request for a server."""
    _fields_ = [("id", c_uint64), ("scene", c_int32), ("camera", Camera), ("width", c_int32), ("height", c_int32),
                ("samples_per_pixel", c_int32), ("d_image", c_void_p), ("d_depth", c_void_p)]


class Completion(ctypes.Structure):
    _fields_ = [("id", c_uint64), ("status", c_int32), ("worker", c_int32), ("queued_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]


class CameraState(ctypes.Structure):
    _fields_ = [
        ("id", c_int32),
        ("width", c_int32),
        ("height", c_int32),
        ("position", c_float * 3),
        ("rotation", c_float * 9),
        ("fx", c_float),
        ("fy", c_float),
        ("img_name", c_char * 64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("num_points_one", c_int32),
        ("num_points_two", c_int32),
        ("num_gaussians_one", c_int32),
        ("num_gaussians_two", c_int32),
        ("survivors_one", c_int32),
        ("survivors_two", c_int32),
        ("total_points_one", c_uint32),
        ("total_points_two", c_uint32),
        ("truncated", c_int32),
        ("device_timeouts", c_int32),
        ("kernel_launches", c_int32),
        ("gaussians_read_one", c_int32),
        ("gaussians_read_two", c_int32),
        ("screen_order_one", c_int32),
        ("screen_order_two", c_int32),
    ]


class DebugView(ctypes.Structure):
    _fields_ = [
        ("counts", c_void_p),
        ("mask_last", c_void_p),
        ("mask_other", c_void_p),
        ("surv_gid", c_void_p),
        ("surv_start", c_void_p),
        ("survivors", c_uint32),
        ("points", c_uint32),
        ("records", c_void_p),
        ("hiz", c_void_p),
        ("hiz_size", c_uint64),
        ("block_culled", c_void_p),
        ("block_words", c_uint32),
        ("block_nodes", c_void_p),
        ("block_count", c_uint32),
        ("per_block", c_uint32),
    ]


# (name, restype, argtypes) for every exported entry point of include/gps_b200.h
_SIGNATURES = [
    ("gps_abi_version", c_int32, []),
    ("gps_last_error", c_char_p, []),
    ("gps_settings_default", None, [POINTER(Settings)]),
    ("gps_settings_parse_args", c_int32, [c_int32, POINTER(c_char_p), POINTER(Settings), c_char_p, ctypes.c_size_t, c_char_p, ctypes.c_size_t]),
    ("gps_scene_load_ply", c_int32, [c_char_p, c_int32, c_int32, POINTER(c_void_p), POINTER(c_int32)]),
    ("gps_scene_from_host", c_int32, [c_void_p, c_uint64, c_int32, c_int32, POINTER(c_void_p)]),
    ("gps_scene_from_host_sorted", c_int32, [c_void_p, c_uint64, c_int32, c_int32, POINTER(c_void_p)]),
    ("gps_morton_order", c_int32, [c_void_p, c_uint64, c_int32, POINTER(c_uint32)]),
    ("gps_scene_tile", c_int32, [c_void_p, c_int32, POINTER(c_float), POINTER(c_void_p)]),
    ("gps_scene_count", c_uint64, [c_void_p]),
    ("gps_scene_format_of", c_int32, [c_void_p]),
    ("gps_scene_free", None, [c_void_p]),
    ("gps_ply_write", c_int32, [c_char_p, c_void_p, c_uint64, c_char_p]),
    ("gps_ply_read", c_int32, [c_char_p, c_void_p, c_uint64, POINTER(c_uint64), POINTER(c_int32)]),
    ("gps_renderer_create", c_int32, [c_void_p, POINTER(Settings), POINTER(c_void_p)]),
    ("gps_renderer_free", None, [c_void_p]),
    ("gps_render_frame", c_int32, [c_void_p, POINTER(Camera), c_void_p, c_void_p, c_void_p]),
    ("gps_renderer_reset", c_int32, [c_void_p, c_void_p]),
    ("gps_renderer_stats", c_int32, [c_void_p, POINTER(Stats)]),
    ("gps_renderer_enable_timing", c_int32, [c_void_p, c_int32]),
    ("gps_renderer_stage_times", c_int32, [c_void_p, POINTER(c_float), POINTER(c_uint64), c_int32]),
    ("gps_renderer_splat_buffer", c_int32, [c_void_p, POINTER(c_void_p), POINTER(c_uint64)]),
    ("gps_renderer_derived", c_int32, [c_void_p, POINTER(Camera), POINTER(c_float)]),
    ("gps_renderer_debug_view", c_int32, [c_void_p, POINTER(DebugView)]),
    ("gps_post_taa", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_float), c_float, c_int32, c_int32, c_int32, c_void_p]),
    ("gps_post_progressive", c_int32, [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p]),
    ("gps_measure_atomic_min_rate", c_int32, [c_void_p, c_uint64, c_int32, POINTER(ctypes.c_double), c_void_p]),
    ("gps_workload_scan_noalloc", c_int32, [c_void_p, c_void_p, c_uint32, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("gps_batch_create", c_int32, [c_void_p, POINTER(Settings), c_int32, c_int32, c_int32, c_int32, POINTER(c_void_p)]),
    ("gps_batch_free", None, [c_void_p]),
    ("gps_batch_render", c_int32, [c_void_p, POINTER(View), c_int32, c_void_p]),
    ("gps_batch_set_workers", c_int32, [c_void_p, c_int32]),
    ("gps_batch_workers", c_int32, [c_void_p]),
    ("gps_batch_autotune", c_int32, [c_void_p, POINTER(View), c_int32, c_int32, c_void_p, POINTER(c_int32), POINTER(c_float)]),
    ("gps_batch_autotune_k", c_int32, [c_void_p, POINTER(View), c_int32, c_int32, c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_float)]),
    ("gps_batch_set_points_per_thread", c_int32, [c_void_p, c_int32]),
    ("gps_batch_use_graph", c_int32, [c_void_p, c_int32]),
    ("gps_batch_graph_stats", c_int32, [c_void_p, POINTER(ctypes.c_int64), POINTER(ctypes.c_int64)]),
    ("gps_server_create", c_int32, [POINTER(c_void_p), c_int32, POINTER(Settings), c_int32, c_int32, c_int32, c_int32, POINTER(c_void_p)]),
    ("gps_server_set_admission", c_int32, [c_void_p, c_uint64]),
    ("gps_server_submit", c_int32, [c_void_p, POINTER(Request)]),
    ("gps_server_poll", c_int32, [c_void_p, POINTER(Completion), c_int32]),
    ("gps_server_drain", c_int32, [c_void_p, ctypes.c_double]),
    ("gps_server_free", None, [c_void_p]),
    ("gps_frame_loop_create", c_int32, [c_void_p, POINTER(c_void_p)]),
    ("gps_frame_loop_free", None, [c_void_p]),
    ("gps_frame_loop_step", c_int32, [c_void_p, POINTER(Camera), c_void_p]),
    ("gps_frame_loop_read", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("gps_frame_loop_read_async", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("gps_frame_loop_read_wait", c_int32, [c_void_p]),
    ("gps_frame_loop_buffers", c_int32, [c_void_p, c_int32, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p)]),
    ("gps_write_png", c_int32, [c_char_p, c_void_p, c_int32, c_int32, c_int32]),
    ("gps_write_pfm", c_int32, [c_char_p, c_void_p, c_int32, c_int32]),
    ("gps_frame_loop_export_pfm", c_int32, [c_void_p, c_char_p, c_void_p]),
    ("gps_evaluate", c_int32, [c_void_p, c_void_p, c_char_p, POINTER(c_int32), c_int32, c_int32, c_int32, c_int32,
                               POINTER(c_int32)]),
    ("gps_camera_path_load", c_int32, [c_char_p, POINTER(c_void_p)]),
    ("gps_camera_path_count", c_int32, [c_void_p]),
    ("gps_camera_path_get", c_int32, [c_void_p, c_int32, POINTER(CameraState)]),
    ("gps_camera_path_free", None, [c_void_p]),
    ("gps_camera_from_state", c_int32, [POINTER(CameraState), POINTER(Settings), c_int32, POINTER(c_int32), c_int32, POINTER(Camera)]),
    ("gps_camera_from_pose", c_int32, [POINTER(c_float), POINTER(c_float), POINTER(Settings), c_int32, POINTER(Camera)]),
]

EXPORTED_SYMBOLS = [s[0] for s in _SIGNATURES]

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libgps_b200.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C {_HERE}` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int):
    if status != 0:
        raise GpsError(status, load_library().gps_last_error().decode(errors="replace"))


def default_settings(**overrides) -> Settings:
    s = Settings()
    load_library().gps_settings_default(byref(s))
    for k, v in overrides.items():
        if k == "background":
            for i in range(3):
                s.background[i] = float(v[i])
        else:
            setattr(s, k, v)
    return s


def parse_args(argv):
    """Mirror of the reference's parseCommandLine (parse_args.cuh:21-127)."""
    s = default_settings()
    arr = (c_char_p * len(argv))(*[a.encode() for a in argv])
    model = ctypes.create_string_buffer(4096)
    cams = ctypes.create_string_buffer(4096)
    _check(load_library().gps_settings_parse_args(len(argv), arr, byref(s), model, 4096, cams, 4096))
    return s, model.value.decode(), cams.value.decode()


def camera_from_pose(position, basis_cols, settings: Settings, frame: int) -> Camera:
    cam = Camera()
    p = (c_float * 3)(*[float(x) for x in position])
    b = (c_float * 9)(*[float(x) for x in np.asarray(basis_cols, dtype=np.float32).reshape(-1)])
    _check(load_library().gps_camera_from_pose(p, b, byref(settings), frame, byref(cam)))
    return cam


def look_at_basis(position, target, up=(0.0, 1.0, 0.0)):
    """Camera-to-world rotation columns (right, down, forward) — the 3DGS / COLMAP convention of
    cameras.json — for a camera at `position` looking at `target`; returned as a (3, 3) array
    whose rows are those columns."""
    p = np.asarray(position, np.float64)
    f = np.asarray(target, np.float64) - p
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return np.stack([r, -u, f], axis=0).astype(np.float32)


def camera_to_numpy(cam: Camera):
    return {
        "view": np.frombuffer(bytes(cam.view), np.float32).copy(),
        "proj": np.frombuffer(bytes(cam.proj), np.float32).copy(),
        "position": np.frombuffer(bytes(cam.position), np.float32).copy(),
        "planes": np.frombuffer(bytes(cam.frustum_planes), np.float32).copy(),
        "frame": cam.frame,
    }


class CameraPath:
    """3DGS cameras.json (camera_loader.cu:123-150)."""

    def __init__(self, path: str):
        self._h = c_void_p()
        _check(load_library().gps_camera_path_load(path.encode(), byref(self._h)))

    def __len__(self):
        return load_library().gps_camera_path_count(self._h)

    def __getitem__(self, i) -> CameraState:
        st = CameraState()
        _check(load_library().gps_camera_path_get(self._h, i, byref(st)))
        return st

    def camera(self, i, settings: Settings, frame: int, override: bool = False, can_override=None):
        cam = Camera()
        can = c_int32(1 if can_override is None else int(can_override))
        st = self[i]
        _check(load_library().gps_camera_from_state(byref(st), byref(settings), int(override), byref(can), frame, byref(cam)))
        return cam, bool(can.value)

    def close(self):
        if self._h:
            load_library().gps_camera_path_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def morton_order(gaussians: np.ndarray, on_device: bool = False) -> np.ndarray:
    """The Morton reorder's permutation (gps_morton_order): order[j] = input index of the j-th."""
    g = np.ascontiguousarray(gaussians, dtype=np.float32)
    assert g.ndim == 2 and g.shape[1] == GAUSSIAN_FLOATS
    order = np.empty(g.shape[0], np.uint32)
    _check(load_library().gps_morton_order(g.ctypes.data, g.shape[0], int(on_device),
                                           order.ctypes.data_as(POINTER(c_uint32))))
    return order


class Scene:
    """Device-resident Gaussian scene (GPUGaussianScene*, gaussian_types.cuh:421-646)."""

    def __init__(self, handle: c_void_p, presorted: bool = False):
        self._h = handle
        self.presorted = presorted

    @classmethod
    def from_ply(cls, path: str, fmt: int = GPS_SCENE_FP32, sort_morton_order: int = 0) -> "Scene":
        """sort_morton_order: 0 file order, 1 Morton reorder on the host, 2 the same reorder on
        the device (gaussian_loader.cu:363-424); a file in BVH order keeps its order."""
        h = c_void_p()
        pre = c_int32(0)
        _check(load_library().gps_scene_load_ply(path.encode(), fmt, int(sort_morton_order), byref(h), byref(pre)))
        return cls(h, bool(pre.value))

    @classmethod
    def from_host(cls, gaussians: np.ndarray, fmt: int = GPS_SCENE_FP32, presorted: bool = True) -> "Scene":
        g = np.ascontiguousarray(gaussians, dtype=np.float32)
        assert g.ndim == 2 and g.shape[1] == GAUSSIAN_FLOATS
        h = c_void_p()
        _check(load_library().gps_scene_from_host(g.ctypes.data, g.shape[0], fmt, int(presorted), byref(h)))
        return cls(h, presorted)

    @classmethod
    def from_host_sorted(cls, gaussians: np.ndarray, fmt: int = GPS_SCENE_FP32, sort_morton_order: int = 2) -> "Scene":
        """A scene in Morton order: 1 reorders on the host, 2 on the device (same order)."""
        g = np.ascontiguousarray(gaussians, dtype=np.float32)
        assert g.ndim == 2 and g.shape[1] == GAUSSIAN_FLOATS
        h = c_void_p()
        _check(load_library().gps_scene_from_host_sorted(g.ctypes.data, g.shape[0], fmt, int(sort_morton_order), byref(h)))
        return cls(h, False)

    def tile(self, offsets_xz) -> "Scene":
        """A half-precision scene of translated copies of this one (gps_scene_tile)."""
        off = np.ascontiguousarray(np.asarray(offsets_xz, np.float32).reshape(-1, 2))
        h = c_void_p()
        _check(load_library().gps_scene_tile(self._h, off.shape[0], off.ctypes.data_as(POINTER(c_float)), byref(h)))
        return Scene(h, self.presorted)

    @property
    def count(self) -> int:
        return int(load_library().gps_scene_count(self._h))

    def close(self):
        if self._h:
            load_library().gps_scene_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ply_write(path: str, gaussians: np.ndarray, comments=()):
    g = np.ascontiguousarray(gaussians, dtype=np.float32)
    c = "\n".join(comments).encode() if comments else None
    _check(load_library().gps_ply_write(path.encode(), g.ctypes.data, g.shape[0], c))


def ply_read(path: str):
    lib = load_library()
    n = c_uint64(0)
    pre = c_int32(0)
    _check(lib.gps_ply_read(path.encode(), None, 0, byref(n), byref(pre)))
    out = np.empty((n.value, GAUSSIAN_FLOATS), np.float32)
    _check(lib.gps_ply_read(path.encode(), out.ctypes.data, n.value, byref(n), byref(pre)))
    return out, bool(pre.value)


class Renderer:
    """GaussianPointSplatting: one render pass object bound to a scene and settings."""

    def __init__(self, scene: Scene, settings: Settings):
        self.scene = scene
        self.settings = settings
        self._h = c_void_p()
        _check(load_library().gps_renderer_create(scene._h, byref(settings), byref(self._h)))

    def render(self, cam: Camera, d_image: int, d_depth: int, stream: int = 0):
        """RenderPass::render into caller-owned device buffers (raw device pointers)."""
        _check(load_library().gps_render_frame(self._h, byref(cam), c_void_p(d_image), c_void_p(d_depth), c_void_p(stream)))

    def reset(self, stream: int = 0):
        """Forget the previous frame: the next render is that of a fresh renderer."""
        _check(load_library().gps_renderer_reset(self._h, c_void_p(stream)))

    def stats(self) -> Stats:
        st = Stats()
        _check(load_library().gps_renderer_stats(self._h, byref(st)))
        return st

    STAGES = ("clear", "block_cull", "preprocess", "scan", "splat", "resolve", "hiz", "post")

    def enable_timing(self, on: bool = True):
        _check(load_library().gps_renderer_enable_timing(self._h, int(on)))

    def stage_times(self, reset: bool = True):
        ms = (c_float * 8)()
        ln = (c_uint64 * 8)()
        _check(load_library().gps_renderer_stage_times(self._h, ms, ln, int(reset)))
        return {k: (float(ms[i]), int(ln[i])) for i, k in enumerate(self.STAGES)}

    def splat_buffer(self):
        p = c_void_p()
        n = c_uint64()
        _check(load_library().gps_renderer_splat_buffer(self._h, byref(p), byref(n)))
        return p.value, n.value

    def derived(self, cam: Camera) -> np.ndarray:
        out = (c_float * 36)()
        _check(load_library().gps_renderer_derived(self._h, byref(cam), out))
        return np.frombuffer(bytes(out), np.float32).copy()

    def debug_view(self) -> DebugView:
        v = DebugView()
        _check(load_library().gps_renderer_debug_view(self._h, byref(v)))
        return v

    def close(self):
        if self._h:
            load_library().gps_renderer_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many views of one scene per call (gps_batch_*): each view bit-identical to a fresh
    single-view render, the views spread over `workers` streams."""

    def __init__(self, scene: Scene, settings: Settings, max_width: int, max_height: int, max_spp: int, workers: int = 4):
        self.scene = scene
        self._h = c_void_p()
        _check(load_library().gps_batch_create(scene._h, byref(settings), max_width, max_height, max_spp, workers,
                                               byref(self._h)))

    @staticmethod
    def views(entries) -> "ctypes.Array":
        """entries: (Camera, width, height, spp, d_image, d_depth) tuples -> gps_view array."""
        arr = (View * len(entries))()
        for i, (cam, w, h, spp, img, dep) in enumerate(entries):
            arr[i] = View(cam, w, h, spp, c_void_p(img), c_void_p(dep))
        return arr

    def render(self, views, stream: int = 0):
        _check(load_library().gps_batch_render(self._h, views, len(views), c_void_p(stream)))

    @property
    def workers(self) -> int:
        return load_library().gps_batch_workers(self._h)

    @workers.setter
    def workers(self, n: int):
        _check(load_library().gps_batch_set_workers(self._h, n))

    def autotune(self, views, rounds: int = 2, stream: int = 0):
        chosen = c_int32()
        ms = c_float()
        _check(load_library().gps_batch_autotune(self._h, views, len(views), rounds, c_void_p(stream), byref(chosen),
                                                 byref(ms)))
        return chosen.value, ms.value

    def autotune_k(self, views, rounds: int = 2, stream: int = 0):
        """K in {1, 2, 4, 8} x worker count; returns (workers, K, ms per batch)."""
        w, k, ms = c_int32(), c_int32(), c_float()
        _check(load_library().gps_batch_autotune_k(self._h, views, len(views), rounds, c_void_p(stream), byref(w), byref(k),
                                                   byref(ms)))
        return w.value, k.value, ms.value

    def set_points_per_thread(self, k: int):
        _check(load_library().gps_batch_set_points_per_thread(self._h, k))

    def use_graph(self, enable: bool = True):
        _check(load_library().gps_batch_use_graph(self._h, int(enable)))

    def graph_stats(self):
        inst, upd = ctypes.c_int64(), ctypes.c_int64()
        _check(load_library().gps_batch_graph_stats(self._h, byref(inst), byref(upd)))
        return inst.value, upd.value

    def close(self):
        if self._h:
            load_library().gps_batch_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop over resident scenes (gps_server_*): submit from any thread, poll completions."""

    def __init__(self, scenes, settings: Settings, max_width: int, max_height: int, max_spp: int, workers: int = 4):
        self.scenes = list(scenes)
        arr = (c_void_p * len(self.scenes))(*[sc._h.value for sc in self.scenes])
        self._h = c_void_p()
        _check(load_library().gps_server_create(arr, len(self.scenes), byref(settings), max_width, max_height, max_spp,
                                                workers, byref(self._h)))

    def submit(self, req_id: int, scene: int, cam: Camera, width: int, height: int, spp: int,
               d_image: int = 0, d_depth: int = 0):
        q = Request(req_id, scene, cam, width, height, spp, c_void_p(d_image or None), c_void_p(d_depth or None))
        _check(load_library().gps_server_submit(self._h, byref(q)))

    def set_admission(self, max_inflight_entries: int):
        """Splat-buffer entries allowed in flight at once (0 = no limit)."""
        _check(load_library().gps_server_set_admission(self._h, max_inflight_entries))

    def poll(self, capacity: int = 256):
        buf = (Completion * capacity)()
        n = load_library().gps_server_poll(self._h, buf, capacity)
        return [(c.id, c.status, c.worker, c.queued_ms, c.latency_ms) for c in buf[:n]]

    def drain(self, timeout_s: float = 600.0):
        _check(load_library().gps_server_drain(self._h, timeout_s))

    def close(self):
        if self._h:
            load_library().gps_server_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FrameLoop:
    """RenderServer::renderFrame without GL (render_server.cu:86-157)."""

    def __init__(self, renderer: Renderer):
        self.renderer = renderer
        self._h = c_void_p()
        _check(load_library().gps_frame_loop_create(renderer._h, byref(self._h)))

    def step(self, cam: Camera, stream: int = 0):
        _check(load_library().gps_frame_loop_step(self._h, byref(cam), c_void_p(stream)))

    def read(self, out: np.ndarray | None = None, stream: int = 0) -> np.ndarray:
        s = self.renderer.settings
        if out is None:
            out = np.empty((s.height, s.width, 3), np.uint8)
        _check(load_library().gps_frame_loop_read(self._h, out.ctypes.data, c_void_p(stream)))
        return out

    def read_async(self, out: np.ndarray, stream: int = 0):
        """Starts copying the last frame to `out` (pinned, untouched until read_wait)."""
        _check(load_library().gps_frame_loop_read_async(self._h, out.ctypes.data, c_void_p(stream)))

    def read_wait(self):
        _check(load_library().gps_frame_loop_read_wait(self._h))

    def buffers(self, slot: int):
        """(u8 image, colour, depth) device pointers of ping-pong slot 0 or 1."""
        u8, col, dep = c_void_p(), c_void_p(), c_void_p()
        _check(load_library().gps_frame_loop_buffers(self._h, slot, byref(u8), byref(col), byref(dep)))
        return u8.value, col.value, dep.value

    def export_pfm(self, path: str, stream: int = 0):
        """The running mean of the last frame's colour buffer as a PFM (export_pfm_from_buffer)."""
        _check(load_library().gps_frame_loop_export_pfm(self._h, path.encode(), c_void_p(stream)))

    def evaluate(self, cameras: "CameraPath", out_dir: str, spp_targets=None, max_eval_count: int = 40,
                 first_frame: int = 0, write_pfm: bool = False) -> int:
        """The evaluation-screenshot run (main.cu:72-120): <out_dir>/<img_name>_spp%04d.png per
        camera and spp target.  Returns the number of frames rendered."""
        tgt, n = None, 0
        if spp_targets is not None:
            n = len(spp_targets)
            tgt = (c_int32 * n)(*spp_targets)
        frames = c_int32(0)
        _check(load_library().gps_evaluate(self._h, cameras._h, out_dir.encode(), tgt, n, max_eval_count,
                                           first_frame, int(write_pfm), byref(frames)))
        return frames.value

    def close(self):
        if self._h:
            load_library().gps_frame_loop_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_png(path: str, rgb: np.ndarray, flip_rows: bool = False):
    """8-bit RGB (H, W, 3) to PNG (stbi_write_png)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    _check(load_library().gps_write_png(path.encode(), rgb.ctypes.data, rgb.shape[1], rgb.shape[0], int(flip_rows)))


def write_pfm(path: str, rgb: np.ndarray):
    """float32 RGB (H, W, 3) to PFM (write_pfm)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    _check(load_library().gps_write_pfm(path.encode(), rgb.ctypes.data, rgb.shape[1], rgb.shape[0]))


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)).astype(np.uint64)
    return x ^ (x >> np.uint64(31))


def buffer_checksum(buf: np.ndarray) -> int:
    """Order-independent 64-bit checksum of a u64 splat buffer (sum of mixed (value, index))."""
    b = np.ascontiguousarray(buf, dtype=np.uint64)
    idx = np.arange(b.size, dtype=np.uint64) * np.uint64(0xD1B54A32D192ED03)
    with np.errstate(over="ignore"):
        return int(np.sum(splitmix64(b ^ idx), dtype=np.uint64))
