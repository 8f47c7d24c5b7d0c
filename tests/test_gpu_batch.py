"""Batched multi-view rendering (gps_batch_*) against plain single-view renders.

A batch renders every view as a fresh renderer's first frame, so each view's image and depth
must be bit-identical to gps_render_frame on a renderer created for that view alone, whatever
the mix of resolutions and samples per pixel, the number of workers or the order of views.
"""
import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

pytestmark = pytest.mark.gpu

RES = [(320, 180), (640, 360), (160, 90), (400, 240)]
SPP = [1, 2, 4, 8]


def _views(n, seed):
    rng = np.random.default_rng(seed)
    poses = synth.random_poses(n, seed=seed)
    out = []
    for i in range(n):
        w, h = RES[int(rng.integers(len(RES)))]
        spp = SPP[int(rng.integers(len(SPP)))]
        out.append((poses[i], w, h, spp, 1 + int(rng.integers(50))))
    return out


def _plain(scene, base, view):
    import torch

    (pose, w, h, spp, frame) = view
    s = gpsplat.default_settings(**base, width=w, height=h, samples_per_pixel=spp)
    cam = gpsutil.cameras_for(s, [pose], first_frame=frame)[0]
    r = gpsplat.Renderer(scene, s)
    img = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    dep = torch.empty((h, w), dtype=torch.float32, device="cuda")
    r.render(cam, img.data_ptr(), dep.data_ptr(), 0)
    torch.cuda.synchronize()
    r.close()
    return cam, img.cpu().numpy(), dep.cpu().numpy()


@pytest.mark.parametrize("occlusion,workers", [(1, 4), (0, 3)])
def test_batch_matches_plain_renders(occlusion, workers):
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    base = dict(supersampling_factor=2, enable_occlusion_culling=occlusion, max_number_of_points=4_000_000)
    views = _views(10, seed=11 + occlusion)
    plain = [_plain(scene, base, v) for v in views]
    s = gpsplat.default_settings(**base, width=640, height=360, samples_per_pixel=8)
    batch = gpsplat.Batch(scene, s, 640, 360, 8, workers=workers)
    bufs = [(torch.full((v[2], v[1], 3), -1.0, device="cuda"), torch.full((v[2], v[1]), -1.0, device="cuda")) for v in views]
    entries = [(plain[i][0], v[1], v[2], v[3], bufs[i][0].data_ptr(), bufs[i][1].data_ptr()) for i, v in enumerate(views)]
    arr = gpsplat.Batch.views(entries)
    for call in range(2):  # twice: worker state left by one batch must not leak into the next
        batch.render(arr)
        torch.cuda.synchronize()
        for i in range(len(views)):
            img, dep = bufs[i][0].cpu().numpy(), bufs[i][1].cpu().numpy()
            assert np.array_equal(img.view(np.uint32), plain[i][1].view(np.uint32)), f"call {call} view {i}: image differs"
            assert np.array_equal(dep.view(np.uint32), plain[i][2].view(np.uint32)), f"call {call} view {i}: depth differs"
    chosen, ms = batch.autotune(arr, rounds=1)
    assert 1 <= chosen <= workers and ms > 0
    batch.close()
    scene.close()


def test_batch_rejects_views_beyond_capacity():
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    s = gpsplat.default_settings(width=320, height=180, samples_per_pixel=2)
    batch = gpsplat.Batch(scene, s, 320, 180, 2, workers=1)
    img = torch.empty((360, 640, 3), device="cuda")
    dep = torch.empty((360, 640), device="cuda")
    cam = gpsutil.cameras_for(s, synth.random_poses(1))[0]
    with pytest.raises(gpsplat.GpsError) as e:
        batch.render(gpsplat.Batch.views([(cam, 640, 360, 2, img.data_ptr(), dep.data_ptr())]))
    assert e.value.status == 6
    batch.close()
    scene.close()


def test_reset_makes_next_frame_a_fresh_render():
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    s = gpsplat.default_settings(width=320, height=180, samples_per_pixel=2, max_number_of_points=4_000_000)
    poses = synth.random_poses(2, seed=3)
    cams = gpsutil.cameras_for(s, poses, first_frame=7)
    _, want_img, want_dep = _plain(scene, dict(max_number_of_points=4_000_000), (poses[1], 320, 180, 2, 8))
    r = gpsplat.Renderer(scene, s)
    img = torch.empty((180, 320, 3), device="cuda")
    dep = torch.empty((180, 320), device="cuda")
    r.render(cams[0], img.data_ptr(), dep.data_ptr(), 0)
    r.reset(0)
    r.render(cams[1], img.data_ptr(), dep.data_ptr(), 0)
    torch.cuda.synchronize()
    assert np.array_equal(img.cpu().numpy().view(np.uint32), want_img.view(np.uint32))
    assert np.array_equal(dep.cpu().numpy().view(np.uint32), want_dep.view(np.uint32))
    r.close()
    scene.close()


def test_frame_loop_async_readback_matches_blocking_read():
    """gps_frame_loop_read_async alternates two u8 frames; the frames it reads back equal the
    blocking read of the same frames on an identical loop."""
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    s = gpsplat.default_settings(width=320, height=180, samples_per_pixel=2, max_number_of_points=4_000_000,
                                 accumulation_mode=gpsplat.GPS_ACCUM_TAA)
    cams = gpsutil.cameras_for(s, synth.orbit(5, 30.0, 10.0))
    ra, rb = gpsplat.Renderer(scene, s), gpsplat.Renderer(scene, s)
    la, lb = gpsplat.FrameLoop(ra), gpsplat.FrameLoop(rb)
    want = []
    for c in cams:
        la.step(c)
        want.append(la.read().copy())
    host = [torch.empty((180, 320, 3), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    for i, c in enumerate(cams):
        lb.step(c)
        lb.read_async(host[i % 2].numpy())
    lb.read_wait()
    n = len(cams)
    assert np.array_equal(host[(n - 1) % 2].numpy(), want[-1])
    assert np.array_equal(host[(n - 2) % 2].numpy(), want[-2])
    for obj in (la, lb, ra, rb, scene):
        obj.close()


@pytest.mark.parametrize("k", [1, 2, 8])
def test_batch_with_points_per_thread_matches_plain_at_same_k(k):
    """K (points_per_thread, not in the reference) moves work between points and samples; a
    batch view rendered with K is bit-identical to a plain render with the same K, and a
    different K gives a different sample stream of the same estimator."""
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    base = dict(supersampling_factor=2, max_number_of_points=4_000_000, points_per_thread=k)
    views = _views(6, seed=40 + k)
    plain = [_plain(scene, base, v) for v in views]
    s = gpsplat.default_settings(**base, width=640, height=360, samples_per_pixel=8)
    batch = gpsplat.Batch(scene, s, 640, 360, 8, workers=2)
    batch.set_points_per_thread(k)
    bufs = [(torch.empty((v[2], v[1], 3), device="cuda"), torch.empty((v[2], v[1]), device="cuda")) for v in views]
    arr = gpsplat.Batch.views([(plain[i][0], v[1], v[2], v[3], bufs[i][0].data_ptr(), bufs[i][1].data_ptr())
                               for i, v in enumerate(views)])
    batch.render(arr)
    torch.cuda.synchronize()
    for i in range(len(views)):
        assert np.array_equal(bufs[i][0].cpu().numpy().view(np.uint32), plain[i][1].view(np.uint32)), f"K={k} view {i}"
        assert np.array_equal(bufs[i][1].cpu().numpy().view(np.uint32), plain[i][2].view(np.uint32)), f"K={k} view {i}"
    # the reference's K (= ss^2 = 4) samples differently but estimates the same image
    ref = _plain(scene, dict(supersampling_factor=2, max_number_of_points=4_000_000), views[0])
    assert not np.array_equal(ref[1], plain[0][1])
    assert abs(float(ref[1].mean()) - float(plain[0][1].mean())) < 0.02
    batch.close()
    scene.close()


def test_batch_graph_replay_matches_direct_launches():
    """The CUDA-graph replay of a batch: the first batch instantiates the graph, a second batch
    with the same layout and new cameras updates it in place; both match plain renders bit for
    bit, and a batch of another layout instantiates a new graph."""
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scene = gpsplat.Scene.from_ply(ply)
    base = dict(supersampling_factor=2, max_number_of_points=4_000_000)
    s = gpsplat.default_settings(**base, width=640, height=360, samples_per_pixel=8)
    batch = gpsplat.Batch(scene, s, 640, 360, 8, workers=3)
    batch.use_graph(True)
    layout = _views(8, seed=70)
    for call, seed in enumerate((71, 72)):
        poses = synth.random_poses(len(layout), seed=seed)
        views = [(poses[i], w, h, spp, frame) for i, (_, w, h, spp, frame) in enumerate(layout)]
        plain = [_plain(scene, base, v) for v in views]
        bufs = [(torch.empty((v[2], v[1], 3), device="cuda"), torch.empty((v[2], v[1]), device="cuda")) for v in views]
        arr = gpsplat.Batch.views([(plain[i][0], v[1], v[2], v[3], bufs[i][0].data_ptr(), bufs[i][1].data_ptr())
                                   for i, v in enumerate(views)])
        batch.render(arr)
        torch.cuda.synchronize()
        for i in range(len(views)):
            assert np.array_equal(bufs[i][0].cpu().numpy().view(np.uint32), plain[i][1].view(np.uint32)), f"call {call} view {i}"
            assert np.array_equal(bufs[i][1].cpu().numpy().view(np.uint32), plain[i][2].view(np.uint32)), f"call {call} view {i}"
    assert batch.graph_stats() == (1, 1), batch.graph_stats()
    other = _views(5, seed=73)
    plain = [_plain(scene, base, v) for v in other]
    bufs = [(torch.empty((v[2], v[1], 3), device="cuda"), torch.empty((v[2], v[1]), device="cuda")) for v in other]
    arr = gpsplat.Batch.views([(plain[i][0], v[1], v[2], v[3], bufs[i][0].data_ptr(), bufs[i][1].data_ptr())
                               for i, v in enumerate(other)])
    batch.render(arr)
    torch.cuda.synchronize()
    assert batch.graph_stats()[0] == 2
    for i in range(len(other)):
        assert np.array_equal(bufs[i][0].cpu().numpy().view(np.uint32), plain[i][1].view(np.uint32))
    w, k, ms = batch.autotune_k(arr, rounds=1)
    assert k in (1, 2, 4, 8) and 1 <= w <= 3 and ms > 0
    batch.close()
    scene.close()
