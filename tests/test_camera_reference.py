"""The camera boundary against the reference's own camera code, bit for bit.

tests/golden/camera_ref.npz holds what the reference computes for every camera of a
cameras.json (`ref_harness camera`: camera_loader.cu:62-90 fromCameraState with its
resolution/fovy override rules, the view matrix of main.cu:141-157, glm::perspective and the
frustum planes of camera.cpp:88-156), for synthetic files and, where present, the reference's
own assets/cameras/*.json.  This library's gps_camera_path_load + gps_camera_from_state must
give the same float bits.  When the reference harness is built in this tree, the synthetic
files are also run through it live.  CPU only.
"""
import glob
import hashlib
import os
import sys

import numpy as np
import pytest

import gpsplat

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_camera_golden as mcg  # noqa: E402

FIXTURE = np.load(os.path.join(HERE, "golden", "camera_ref.npz"))


def _mine(json_path, row):
    """Replays the viewer's sequence: load_camera() selects camera 0 (which may take the
    resolution from the file), then every camera in turn (render_settings.cuh:233-256)."""
    w, h, fovy, near, far, override = row
    s = gpsplat.default_settings(width=int(w), height=int(h), fovy=float(fovy), near_view_plane=float(near),
                                 far_view_plane=float(far))
    path = gpsplat.CameraPath(json_path)
    _, can = path.camera(0, s, frame=1, override=bool(override), can_override=True)
    mats, res = [], []
    for i in range(min(len(path), mcg.MAX_CAMERAS)):
        cam, can = path.camera(i, s, frame=1 + i, override=bool(override), can_override=can)
        d = gpsplat.camera_to_numpy(cam)
        mats.append(np.concatenate([d["view"], d["proj"], d["planes"], d["position"],
                                    np.array([s.fovy], np.float32)]))
        res.append((s.width, s.height))
    path.close()
    return np.array(mats, np.float32), np.array(res, np.int32)


def _compare(tag, json_path, i, row, ref_mats, ref_res):
    mats, res = _mine(json_path, row)
    assert res.shape == ref_res.shape and np.array_equal(res, ref_res), f"{tag} row {i}: resolution differs"
    names = [("view", 0, 16), ("proj", 16, 32), ("planes", 32, 56), ("position", 56, 59), ("fovy", 59, 60)]
    for name, a, b in names:
        mine = mats[:, a:b].view(np.uint32)
        ref = ref_mats[:, a:b].view(np.uint32)
        bad = np.nonzero(np.any(mine != ref, axis=1))[0]
        assert bad.size == 0, f"{tag} row {i}: {name} differs for cameras {bad[:8]} (first: {mats[bad[0], a:b]} vs {ref_mats[bad[0], a:b]})"


@pytest.fixture(scope="module")
def synthetic_files(tmp_path_factory):
    return mcg.synthetic_json_files(str(tmp_path_factory.mktemp("camjson")))


@pytest.mark.parametrize("tag", ["syn_orbit", "syn_random", "syn_portrait"])
@pytest.mark.parametrize("row", range(len(mcg.SETTINGS)))
def test_synthetic_camera_paths_match_the_reference(synthetic_files, tag, row):
    path = synthetic_files[tag]
    sha = np.frombuffer(hashlib.sha256(open(path, "rb").read()).digest(), np.uint8)
    assert np.array_equal(sha, FIXTURE[f"{tag}__sha256"]), "synthetic cameras.json no longer regenerates identically"
    _compare(tag, path, row, mcg.SETTINGS[row], FIXTURE[f"{tag}__{row}__mats"], FIXTURE[f"{tag}__{row}__res"])
    if os.path.exists(mcg.HARNESS):  # and the reference's camera code itself, live
        mats, res = mcg.run_harness(path, mcg.SETTINGS[row])
        _compare(tag + " (live)", path, row, mcg.SETTINGS[row], mats[:mcg.MAX_CAMERAS], res[:mcg.MAX_CAMERAS])


def _asset_files():
    by_hash = {}
    for p in sorted(glob.glob(os.path.join(mcg.REF_ROOT, "assets", "cameras", "*.json"))):
        by_hash[hashlib.sha256(open(p, "rb").read()).hexdigest()] = p
    out = []
    for key in FIXTURE.files:
        if key.startswith("asset_") and key.endswith("__sha256"):
            out.append((key[:-len("__sha256")], by_hash.get(FIXTURE[key].tobytes().hex())))
    return out


@pytest.mark.parametrize("tag,path", _asset_files())
def test_reference_camera_assets_match_the_reference(tag, path):
    if path is None:
        pytest.skip("the reference's camera assets are not present on this machine")
    for row in range(len(mcg.SETTINGS)):
        _compare(tag, path, row, mcg.SETTINGS[row], FIXTURE[f"{tag}__{row}__mats"], FIXTURE[f"{tag}__{row}__res"])
