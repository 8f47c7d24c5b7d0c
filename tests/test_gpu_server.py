"""The request server (gps_server_*): requests over two resident scenes, submitted while others
are on the GPU, each completed with the same image and depth as a fresh single-view render of
the same request alone; requests beyond the workers' capacity complete with GPS_ERR_SIZE."""
import threading

import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

pytestmark = pytest.mark.gpu

RES = [(320, 180), (640, 360), (160, 90)]
SPP = [1, 4, 2]


def test_server_results_match_plain_renders():
    import torch

    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    scenes = [gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_FP32), gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_HALF)]
    base = dict(supersampling_factor=2, max_number_of_points=4_000_000)
    rng = np.random.default_rng(9)
    poses = synth.random_poses(16, seed=9)
    reqs = []
    for i, pose in enumerate(poses):
        w, h = RES[int(rng.integers(len(RES)))]
        spp = SPP[int(rng.integers(len(SPP)))]
        s = gpsplat.default_settings(**base, width=w, height=h, samples_per_pixel=spp)
        cam = gpsutil.cameras_for(s, [pose], first_frame=1 + i)[0]
        reqs.append(dict(id=100 + i, scene=i % 2, cam=cam, w=w, h=h, spp=spp, s=s,
                         img=torch.full((h, w, 3), -1.0, device="cuda"), dep=torch.full((h, w), -1.0, device="cuda")))
    cap = gpsplat.default_settings(**base, width=640, height=360, samples_per_pixel=4)
    server = gpsplat.Server(scenes, cap, 640, 360, 4, workers=3)
    # submit from another thread in two bursts, the second while the first is in flight
    def producer():
        for q in reqs:
            server.submit(q["id"], q["scene"], q["cam"], q["w"], q["h"], q["spp"], q["img"].data_ptr(), q["dep"].data_ptr())
    t = threading.Thread(target=producer)
    t.start()
    t.join()
    too_big = gpsutil.cameras_for(gpsplat.default_settings(**base, width=1280, height=720), [poses[0]])[0]
    server.submit(999, 0, too_big, 1280, 720, 1)
    server.drain(120.0)
    done = {c[0]: c for c in server.poll(64)}
    assert set(done) == {q["id"] for q in reqs} | {999}
    assert done[999][1] == 6
    for q in reqs:
        assert done[q["id"]][1] == 0
        assert done[q["id"]][4] >= done[q["id"]][3] >= 0.0
        r = gpsplat.Renderer(scenes[q["scene"]], q["s"])
        img = torch.empty_like(q["img"])
        dep = torch.empty_like(q["dep"])
        r.render(q["cam"], img.data_ptr(), dep.data_ptr(), 0)
        torch.cuda.synchronize()
        assert torch.equal(img.view(torch.int32), q["img"].view(torch.int32)), f"request {q['id']}: image differs"
        assert torch.equal(dep.view(torch.int32), q["dep"].view(torch.int32)), f"request {q['id']}: depth differs"
        r.close()
    assert len({c[2] for c in done.values()}) > 1, "requests should spread over several workers"
    server.close()
    for sc in scenes:
        sc.close()
