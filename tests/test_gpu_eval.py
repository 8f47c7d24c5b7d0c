"""The evaluation-screenshot run (gps_evaluate, main.cu:72-120 and render_server.cu:269-315).

gps_evaluate must write, for cameras 0 .. min(count - 1, max_eval_count), the u8 frame after
each spp target of progressive frames as a row-flipped PNG named <img_name>_spp%04d.png, and
those images must be exactly the frames a frame loop driven by hand with the same cameras and
frame numbers produces.  The optional PFM holds the running mean of the colour buffer.
"""
import os

import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

pytestmark = pytest.mark.gpu

W, H = 160, 90


def test_evaluate_writes_the_frames_a_hand_driven_loop_renders(tmp_path):
    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    s = gpsplat.default_settings(width=W, height=H, samples_per_pixel=2, max_number_of_points=4_000_000)
    cams_json = str(tmp_path / "cameras.json")
    synth.write_cameras_json(cams_json, synth.orbit(3, 30.0, 10.0), 1600, 900, 1100.0)
    path = gpsplat.CameraPath(cams_json)
    targets = [1, 2, 4]
    out = str(tmp_path / "eval" / "town")
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    frames = loop.evaluate(path, out, spp_targets=targets, max_eval_count=1, first_frame=5, write_pfm=True)
    assert frames == 2 * 4  # cameras 0 and 1 (the stopping rule: c >= max_eval_count), 4 frames each
    names = sorted(os.listdir(out))
    want = sorted(f"frame_{c:04d}_spp{t:04d}.{ext}" for c in range(2) for t in targets for ext in ("png", "pfm"))
    assert names == want

    r2 = gpsplat.Renderer(scene, s)
    hand = gpsplat.FrameLoop(r2)
    frame = 5
    for c in range(2):
        for f in range(1, 5):
            cam, _ = path.camera(c, gpsplat.default_settings(width=W, height=H, samples_per_pixel=2), frame,
                                 can_override=False)
            cam.camera_moved = int(f == 1)
            hand.step(cam)
            frame += 1
            if f in targets:
                stem = os.path.join(out, f"frame_{c:04d}_spp{f:04d}")
                png = gpsutil.decode_png(open(stem + ".png", "rb").read())
                assert np.array_equal(png, hand.read()[::-1]), (c, f)
                pfm = open(stem + ".pfm", "rb").read()
                head = f"PF\n{W} {H}\n-1.0\n".encode()
                assert pfm.startswith(head)
                mean = np.frombuffer(pfm[len(head):], "<f4").reshape(H, W, 3)
                hand.export_pfm(str(tmp_path / "hand.pfm"))
                assert open(str(tmp_path / "hand.pfm"), "rb").read() == pfm
                # the u8 frame is the same running mean, clamped and rounded (memory order, unflipped)
                u8 = np.clip(np.rint(mean.astype(np.float64) * 255.0), 0, 255)
                assert np.abs(u8 - hand.read().astype(np.float64)).max() <= 1.0
    with pytest.raises(gpsplat.GpsError) as e:
        loop.evaluate(path, out, spp_targets=[4, 2])
    assert e.value.status == 1
    for obj in (hand, r2, loop, r, path, scene):
        obj.close()


def test_evaluate_matches_the_reference_frames(tmp_path):
    """The evaluation run's PNGs against the reference's own kernels and post-process (the
    headless harness, RenderServer::renderFrame's progressive accumulation) fed the same
    cameras, frame numbers and camera-moved flags: every written image is the reference's u8
    frame of that step, row-flipped as save_image_to_disk writes it."""
    if gpsutil.ref_harness("fp32") is None:
        pytest.skip("reference harness not built (oracle/ref/build_ref.sh)")
    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    s = gpsplat.default_settings(width=W, height=H, samples_per_pixel=2, max_number_of_points=4_000_000)
    cams_json = str(tmp_path / "cameras.json")
    synth.write_cameras_json(cams_json, synth.orbit(3, 30.0, 10.0), 1600, 900, 1100.0)
    path = gpsplat.CameraPath(cams_json)
    targets = [1, 2, 4]
    out = str(tmp_path / "eval" / "town")
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    assert loop.evaluate(path, out, spp_targets=targets, max_eval_count=1, first_frame=5) == 8
    cams, frame = [], 5
    for c in range(2):
        for f in range(1, 5):
            cam, _ = path.camera(c, gpsplat.default_settings(width=W, height=H, samples_per_pixel=2), frame,
                                 can_override=False)
            cam.camera_moved = int(f == 1)
            cams.append(cam)
            frame += 1
    ref, _ = gpsutil.run_reference(ply, s, cams)
    for c in range(2):
        for f in targets:
            png = gpsutil.decode_png(open(os.path.join(out, f"frame_{c:04d}_spp{f:04d}.png"), "rb").read())
            assert np.array_equal(png, ref[c * 4 + f - 1]["post_u8"][::-1]), (c, f)
    for obj in (loop, r, path, scene):
        obj.close()
