"""The --sort-morton-order scene reorder (gaussian_loader.cu:363-424).

The library reorders on the host (the reference's own host keys) or on the device (keys, a
stable radix sort and a gather in HBM); both must give the reference's permutation exactly,
ties included, because every later stage indexes Gaussians by their position in the scene.
CPU tests pin the host path to the oracle's restatement; GPU tests pin the device path to the
host path, the reordered scene to the one the reference's own loader builds from the same PLY,
and the renders of host- and device-reordered scenes to each other bit for bit.
"""
import os
import sys

import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

sys.path.insert(0, os.path.join(gpsutil.ROOT, "oracle"))
import oracle  # noqa: E402


def _shuffled(raw, seed):
    perm = np.random.default_rng(seed).permutation(raw.n)
    out = raw.subset(perm)
    out.sorted_order = False
    return out


def _scenes():
    """Activated host scenes that cover the key's edge cases."""
    out = {}
    out["cube_shuffled"] = synth.activate(_shuffled(synth.cube(5000, seed=3), 1))
    g = synth.activate(_shuffled(synth.cube(3000, seed=4), 2))
    g[1000:1500, 0:3] = g[0:500, 0:3]  # equal means: equal keys keep input order
    out["ties"] = g
    g = synth.activate(_shuffled(synth.cube(2000, seed=5), 3))
    g[:, 1] = 2.5  # one flat axis: max - min = 0, that axis's bits are all 0
    out["flat_axis"] = g
    g = synth.activate(_shuffled(synth.cube(2000, seed=6), 4))
    g[:, 0:3] = g[:, 0:3] * np.float32(1e-3) - np.float32(7.0)  # tiny extent, negative coordinates
    out["tiny_negative"] = g
    out["single"] = synth.activate(synth.cube(16, seed=7))[:1]
    out["two_equal"] = np.repeat(synth.activate(synth.cube(16, seed=8))[:1], 2, axis=0)
    return out


SCENES = _scenes()


def test_oracle_key_spot_values():
    """Hand-worked keys: min corner -> 0; the max corner -> all 63 bits; x alone fills bits 3b."""
    g = np.zeros((3, 59), np.float32)
    g[0, 0:3] = (1.0, 1.0, 1.0)  # max corner
    g[1, 0:3] = (0.0, 0.0, 0.0)  # min corner
    g[2, 0:3] = (1.0, 0.0, 0.0)  # x only: key 0o111...1 (every third bit)
    assert oracle.morton_order(g).tolist() == [1, 2, 0]


@pytest.mark.parametrize("name", sorted(SCENES))
def test_host_order_matches_oracle(name):
    g = SCENES[name]
    assert np.array_equal(gpsplat.morton_order(g, on_device=False), oracle.morton_order(g))


def test_host_order_with_nan_means_matches_oracle():
    """A NaN coordinate never wins the bounds' comparisons and its key bits are 0 (the 21 low
    bits of the conversion of NaN), as in the reference's host code."""
    g = synth.activate(_shuffled(synth.cube(3000, seed=12), 8))
    g[5, 0] = np.nan
    g[100, 1:3] = np.nan
    assert np.array_equal(gpsplat.morton_order(g, on_device=False), oracle.morton_order(g))


def test_empty_scene_order():
    g = np.zeros((0, 59), np.float32)
    assert gpsplat.morton_order(g, on_device=False).size == 0
    assert oracle.morton_order(g).size == 0


def test_bad_sort_mode_is_rejected():
    g = SCENES["single"]
    with pytest.raises(gpsplat.GpsError):
        gpsplat.Scene.from_host_sorted(g, gpsplat.GPS_SCENE_FP32, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_order_matches_host(name):
    g = SCENES[name]
    assert np.array_equal(gpsplat.morton_order(g, on_device=True), gpsplat.morton_order(g, on_device=False))


@pytest.mark.gpu
def test_device_order_matches_host_at_scale():
    """2M Gaussians of the town scene, shuffled: many equal keys at 21 bits per axis."""
    g = synth.activate(_shuffled(synth.town(2_000_000, seed=9), 5))
    dev = gpsplat.morton_order(g, on_device=True)
    assert np.array_equal(dev, gpsplat.morton_order(g, on_device=False))
    assert np.array_equal(dev, oracle.morton_order(g))


def _render(scene, s, cams):
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    out = []
    for cam in cams:
        loop.step(cam)
        gpsutil.sync()
        bptr, entries = r.splat_buffer()
        out.append(gpsutil.d2h(bptr, entries, np.uint64))
    loop.close()
    r.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [gpsplat.GPS_SCENE_FP32, gpsplat.GPS_SCENE_HALF, gpsplat.GPS_SCENE_COMPRESSED])
def test_device_reordered_scene_renders_like_host_reordered(fmt):
    g = synth.activate(_shuffled(synth.town(200_000, seed=10), 6))
    s = gpsplat.default_settings(width=640, height=360, supersampling_factor=2, samples_per_pixel=2)
    cams = gpsutil.cameras_for(s, synth.orbit(2, 30.0, 10.0))
    host = gpsplat.Scene.from_host_sorted(g, fmt, 1)
    dev = gpsplat.Scene.from_host_sorted(g, fmt, 2)
    plain = gpsplat.Scene.from_host(g[oracle.morton_order(g)], fmt, presorted=False)
    a, b, c = _render(host, s, cams), _render(dev, s, cams), _render(plain, s, cams)
    for f in range(len(cams)):
        assert np.array_equal(a[f], b[f]), f"frame {f}: device reorder renders differently"
        assert np.array_equal(a[f], c[f]), f"frame {f}: reorder differs from the oracle's order"


@pytest.mark.gpu
@pytest.mark.parametrize("sort_mode", [1, 2])
def test_reorder_matches_reference_loader(sort_mode):
    """The reference's loader (its --sort-morton-order branch, run by the harness on the same
    PLY) against gps_scene_load_ply with the host (1) and device (2) reorder: the reordered
    scenes' splat buffers agree bit for bit, and the reference's reordered host scene is the
    input permuted by the oracle's order."""
    if gpsutil.ref_harness("fp32") is None:
        pytest.skip("reference harness not built (oracle/ref/build_ref.sh)")
    raw = _shuffled(synth.town(100_000, seed=11), 7)
    ply = gpsutil.cached_ply("town100k_shuffled", lambda: raw)
    s = gpsplat.default_settings(width=640, height=360, supersampling_factor=1, samples_per_pixel=1,
                                 sort_morton_order=1)
    cams = gpsutil.cameras_for(s, synth.orbit(1, 30.0, 10.0))
    ref, extra = gpsutil.run_reference(ply, s, cams)
    g, presorted = gpsplat.ply_read(ply)
    assert not presorted
    assert np.array_equal(extra["scene_cpu"], g[oracle.morton_order(g)])
    scene = gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_FP32, sort_morton_order=sort_mode)
    mine = gpsutil.run_mine(scene, s, cams)
    assert np.array_equal(ref[0]["buffer"], mine[0]["buffer"])
