"""Host-side boundary of the library (no GPU needed): the C-ABI loads and exports every entry
point include/gps_b200.h declares; settings defaults and CLI parsing mirror the reference's
RenderSettings / parseCommandLine (src/render_settings.cuh:36-103, src/parse_args.cuh:21-127);
the 3DGS PLY reader/writer (src/core/gaussians/gaussian_loader.cu:115-562) and the camera
JSON loader (src/utils/camera_loader.cu:123-150) accept what the reference accepts and fail
with a status (never a crash) on malformed input."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gps_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gps_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = gpsplat.load_library()
    declared = header_functions()
    assert len(declared) >= 30
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, f"declared but not exported: {missing}"
    assert sorted(gpsplat.EXPORTED_SYMBOLS) == declared, "binding and header disagree"
    assert lib.gps_abi_version() == 1


def test_settings_defaults_match_reference():
    s = gpsplat.default_settings()
    assert (s.width, s.height) == (1920, 1080)
    assert s.supersampling_factor == 2 and s.samples_per_pixel == 1
    assert s.max_number_of_points == 250000000
    assert s.fovy == pytest.approx(45.0) and s.near_view_plane == pytest.approx(0.2)
    assert s.far_view_plane == pytest.approx(10000.0)
    assert s.enable_hierarchical_culling == 1 and s.fully_disable_hierarchical_culling == 0
    assert s.enable_occlusion_culling == 1 and s.occlusion_culling_min_reduce_count == 0
    assert s.use_unbiased_2d_splatting == 1 and s.reduce_point_count == 1 and s.cull_small_gaussians == 0
    assert list(s.background) == [0.0, 0.0, 0.0]
    assert s.accumulation_mode == gpsplat.GPS_ACCUM_PROGRESSIVE


def test_parse_args_mirrors_reference_flags():
    s, model, cams = gpsplat.parse_args([
        "viewer", "--model-path", "/data/m", "--camera-path", "/data/c.json", "--resolution", "1280", "720",
        "--supersampling-factor", "3", "--samples-per-pixel", "8", "--max-number-of-points", "1000",
        "--fovy", "60", "--near-view-plane", "0.5", "--far_view_plane", "500", "--one-point-per-thread",
        "--disable-hierarchical-culling", "--disable_occlusion_culling", "--cull-small", "--background", "0.1", "0.2",
        "0.3", "--taa", "--sort-morton-order", "--disable-gui", "--unknown-flag"])
    assert model == "/data/m" and cams == "/data/c.json"
    assert (s.width, s.height, s.supersampling_factor, s.samples_per_pixel) == (1280, 720, 3, 8)
    assert s.max_number_of_points == 1000 and s.fovy == pytest.approx(60.0)
    assert s.near_view_plane == pytest.approx(0.5) and s.far_view_plane == pytest.approx(500.0)
    assert s.reduce_point_count == 0 and s.enable_hierarchical_culling == 0 and s.enable_occlusion_culling == 0
    assert s.cull_small_gaussians == 1 and s.accumulation_mode == gpsplat.GPS_ACCUM_TAA and s.sort_morton_order == 1
    assert [round(v, 3) for v in s.background] == [0.1, 0.2, 0.3]


def test_parse_args_bad_number_is_an_error():
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.parse_args(["viewer", "--samples-per-pixel", "many"])
    assert e.value.status == 1


def test_ply_roundtrip_and_activation(tmp_path):
    raw = synth.cube(500, seed=4)
    p = str(tmp_path / "scene.ply")
    raw.write_ply(p)
    g, pre = gpsplat.ply_read(p)
    assert g.shape == (500, 59) and not pre
    act = synth.activate(raw)
    np.testing.assert_allclose(g, act, rtol=1e-6, atol=1e-6)
    # positions, DC and zero-filled higher SH are copied exactly
    assert np.array_equal(g[:, 0:3], raw.pos)
    assert np.array_equal(g[:, 3:6], raw.dc)
    assert not g[:, 6:51].any()
    # rotations are normalised, opacities are in [0, 1]
    np.testing.assert_allclose(np.linalg.norm(g[:, 55:59], axis=1), 1.0, atol=1e-6)
    assert (g[:, 51] >= 0).all() and (g[:, 51] <= 1).all()
    # the writer emits the reference's full layout (with normals); reading it back is stable
    p2 = str(tmp_path / "again.ply")
    gpsplat.ply_write(p2, g, ["bvh_sorted_order"])
    g2, pre2 = gpsplat.ply_read(p2)
    assert pre2
    np.testing.assert_allclose(g2, g, rtol=2e-5, atol=2e-6)


def test_ply_read_spans_chunks(tmp_path):
    """The reader converts 64 MiB of records at a time while the next chunk is read: a file of
    several chunks reads back like the activation of its fields, and one cut inside a later
    chunk is a short read (GPS_ERR_IO)."""
    raw = synth.cube(700_000, seed=6)  # 248-byte records: three chunks
    p = str(tmp_path / "big.ply")
    raw.write_ply(p)
    g, _ = gpsplat.ply_read(p)
    np.testing.assert_allclose(g, synth.activate(raw), rtol=1e-6, atol=1e-6)
    assert np.array_equal(g[:, 0:3], raw.pos)
    data = open(p, "rb").read()
    cut = str(tmp_path / "cut.ply")
    with open(cut, "wb") as f:
        f.write(data[: len(data) - 200 * 248])
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.ply_read(cut)
    assert e.value.status == 2


def test_ply_sh_rest_is_channel_major(tmp_path):
    raw = synth.town(300, seed=2)
    p = str(tmp_path / "town.ply")
    raw.write_ply(p)
    g, pre = gpsplat.ply_read(p)
    assert pre, "the town generator marks its Morton order as bvh_sorted_order"
    for j in range(1, 16):
        for c in range(3):
            assert np.array_equal(g[:, 3 + 3 * j + c], raw.rest[:, (j - 1) + 15 * c])


def test_ply_property_order_and_extra_fields(tmp_path):
    # header-driven offsets: reorder the properties and add unknown ones
    n = 64
    rng = np.random.default_rng(0)
    names = ["opacity", "rot_3", "x", "junk_a", "f_dc_1", "scale_2", "y", "rot_0", "z", "f_dc_0", "scale_0", "rot_1",
             "f_dc_2", "scale_1", "rot_2"]
    vals = rng.standard_normal((n, len(names))).astype(np.float32)
    p = str(tmp_path / "shuffled.ply")
    with open(p, "wb") as f:
        f.write(("ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n).encode())
        for nm in names:
            f.write(f"property float {nm}\n".encode())
        f.write(b"end_header\n")
        f.write(vals.tobytes())
    g, _ = gpsplat.ply_read(p)
    col = {nm: vals[:, i] for i, nm in enumerate(names)}
    assert np.array_equal(g[:, 0], col["x"]) and np.array_equal(g[:, 1], col["y"]) and np.array_equal(g[:, 2], col["z"])
    assert np.array_equal(g[:, 3], col["f_dc_0"]) and np.array_equal(g[:, 5], col["f_dc_2"])
    q = np.stack([col["rot_0"], col["rot_1"], col["rot_2"], col["rot_3"]], 1)
    np.testing.assert_allclose(g[:, 55:59], q / np.linalg.norm(q, axis=1, keepdims=True), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("body,status", [
    (b"not a ply file\n", 3),
    (b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n", 3),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 0\nproperty float x\nend_header\n", 3),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float x\nproperty float y\nend_header\n", 3),
])
def test_malformed_ply_is_rejected(tmp_path, body, status):
    p = str(tmp_path / "bad.ply")
    with open(p, "wb") as f:
        f.write(body)
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.ply_read(p)
    assert e.value.status == status


def test_truncated_ply_is_an_io_error(tmp_path):
    raw = synth.cube(100, seed=1)
    p = str(tmp_path / "t.ply")
    raw.write_ply(p)
    data = open(p, "rb").read()
    with open(p, "wb") as f:
        f.write(data[:-100])
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.ply_read(p)
    assert e.value.status == 2


def test_missing_file_is_an_io_error(tmp_path):
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.ply_read(str(tmp_path / "nope.ply"))
    assert e.value.status == 2


def test_3dgs_output_directory_resolves_to_last_iteration(tmp_path):
    raw = synth.cube(50, seed=6)
    for it in ("iteration_7000", "iteration_30000", "iteration_000"):
        d = tmp_path / "model" / "point_cloud" / it
        d.mkdir(parents=True)
    # alphabetically last folder wins (render_settings.cuh:166-176)
    raw.write_ply(str(tmp_path / "model" / "point_cloud" / "iteration_7000" / "point_cloud.ply"))
    g, _ = gpsplat.ply_read(str(tmp_path / "model"))
    assert g.shape[0] == 50
    with pytest.raises(gpsplat.GpsError):
        gpsplat.ply_read(str(tmp_path / "model" / "point_cloud"))


def test_camera_path_json(tmp_path):
    poses = synth.orbit(5, 30.0, 10.0)
    p = str(tmp_path / "cameras.json")
    synth.write_cameras_json(p, poses, 4946, 3286, 4627.3, 4649.5)
    # shuffle the order: the loader sorts by id (camera_loader.cu:143-146)
    cams = json.load(open(p))
    json.dump(cams[::-1], open(p, "w"))
    cp = gpsplat.CameraPath(p)
    assert len(cp) == 5
    st = cp[2]
    assert st.id == 2 and st.width == 4946 and st.height == 3286
    assert st.img_name.decode() == "frame_0002"
    np.testing.assert_allclose(list(st.position), poses[2][0], rtol=1e-6)
    np.testing.assert_allclose(np.array(list(st.rotation)).reshape(3, 3), poses[2][1], rtol=1e-5, atol=1e-6)
    # resolution / fovy override rules of fromCameraState (camera_loader.cu:62-90)
    s = gpsplat.default_settings()
    cam, can = cp.camera(2, s, frame=3)
    assert (s.width, s.height) == (1920, int(round(1920 * 3286 / 4946)))
    assert not can
    fov = 2.0 * np.degrees(np.arctan(0.5 * 3286 / 4627.3))
    assert s.fovy == pytest.approx(fov, rel=1e-5)
    assert cam.frame == 3
    # an explicit --resolution / --fovy keeps the settings (override_camera_settings)
    s2 = gpsplat.default_settings(width=800, height=600, fovy=50.0)
    cp.camera(0, s2, frame=1, override=True)
    assert (s2.width, s2.height) == (800, 600) and s2.fovy == pytest.approx(50.0)


@pytest.mark.parametrize("text", ["{not json", "{}", '[{"id": 0}]', '[{"id": 0, "img_name": "a", "width": 1, "height": 1, '
                                  '"position": [0,0], "rotation": [[1,0,0],[0,1,0],[0,0,1]], "fx": 1, "fy": 1}]'])
def test_bad_camera_json_is_a_format_error(tmp_path, text):
    p = str(tmp_path / "c.json")
    open(p, "w").write(text)
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.CameraPath(p)
    assert e.value.status == 3


def test_camera_matrices_follow_the_viewer_conventions():
    s = gpsplat.default_settings(width=640, height=360)
    p = np.array([0.0, 0.0, -30.0])
    cam = gpsplat.camera_from_pose(p, synth.look_at_c2w(p, [0, 0, 0]).T, s, 1)
    d = gpsplat.camera_to_numpy(cam)
    view = d["view"].reshape(4, 4).T
    proj = d["proj"].reshape(4, 4).T
    # the origin is 30 units in front of the camera (OpenGL view space looks down -z)
    np.testing.assert_allclose(view @ np.array([0, 0, 0, 1.0]), [0, 0, -30, 1], atol=1e-5)
    # glm::perspective(fovy, aspect, near, far), NDC z in [-1, 1]
    t = np.tan(np.radians(45.0) / 2)
    np.testing.assert_allclose(proj[1, 1], 1 / t, rtol=1e-6)
    np.testing.assert_allclose(proj[0, 0], 1 / (t * 640 / 360), rtol=1e-6)
    np.testing.assert_allclose(proj[2, 2], -(10000 + 0.2) / (10000 - 0.2), rtol=1e-6)
    planes = d["planes"].reshape(6, 4)
    np.testing.assert_allclose(np.linalg.norm(planes[:, :3], axis=1), 1.0, atol=1e-6)
    # the origin is inside all six frustum planes
    assert (planes[:, 3] > 0).all()


def test_invalid_renderer_settings_are_rejected_without_gpu():
    lib = gpsplat.load_library()
    r = ctypes.c_void_p()
    s = gpsplat.default_settings(width=0)
    assert lib.gps_renderer_create(None, ctypes.byref(s), ctypes.byref(r)) == 1
    assert lib.gps_render_frame(None, None, None, None, None) == 1
    assert lib.gps_post_taa(None, None, None, None, None, None, None, 0.9, 1, 1, 1, None) == 1


def test_png_writer_roundtrip_and_flip(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, size=(37, 53, 3), dtype=np.uint8)
    p = str(tmp_path / "a.png")
    gpsplat.write_png(p, img)
    assert np.array_equal(gpsutil.decode_png(open(p, "rb").read()), img)
    gpsplat.write_png(p, img, flip_rows=True)  # save_image_to_disk's row swap
    assert np.array_equal(gpsutil.decode_png(open(p, "rb").read()), img[::-1])
    with pytest.raises(gpsplat.GpsError) as e:
        gpsplat.write_png(str(tmp_path / "missing_dir" / "a.png"), img)
    assert e.value.status == 2


def test_pfm_writer_layout(tmp_path):
    img = np.arange(4 * 6 * 3, dtype=np.float32).reshape(4, 6, 3) / 7.0
    p = str(tmp_path / "a.pfm")
    gpsplat.write_pfm(p, img)
    data = open(p, "rb").read()
    head = b"PF\n6 4\n-1.0\n"
    assert data[:len(head)] == head
    assert np.array_equal(np.frombuffer(data[len(head):], "<f4").reshape(4, 6, 3), img)
