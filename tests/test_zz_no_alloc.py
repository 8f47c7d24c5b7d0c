"""The allocation-free point scan (gps_workload_scan_noalloc) against the renderer's own scan.

That entry point exists for callers that must not allocate device memory when they run the
scan — a CUDA-graph capture, a host with a fixed device-memory budget, a plugin whose host owns
every buffer — so it keeps its only scratch (the scan's per-tile totals) in a fixed array
inside the library.  This test renders a frame through the normal entry point, then runs the
allocation-free scan twice in a row on that frame's counts and survivor mask, and checks both
results against the workload the renderer computed (integer data: exact).  The file sorts
last so that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("occlusion", [0, 1])
def test_noalloc_scan_matches_renderer_twice(occlusion):
    import torch

    lib = gpsplat.load_library()
    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    s = gpsplat.default_settings(width=320, height=180, supersampling_factor=2, samples_per_pixel=2,
                                 enable_occlusion_culling=occlusion, max_number_of_points=20000)
    cams = gpsutil.cameras_for(s, synth.orbit(2, 30.0, 10.0))
    scene = gpsplat.Scene.from_ply(ply)
    r = gpsplat.Renderer(scene, s)
    img = torch.zeros((s.height, s.width, 3), dtype=torch.float32, device="cuda")
    dep = torch.zeros((s.height, s.width), dtype=torch.float32, device="cuda")
    for cam in cams:
        r.render(cam, img.data_ptr(), dep.data_ptr(), 0)
    torch.cuda.synchronize()
    v = r.debug_view()
    n = scene.count
    want_gid = gpsutil.d2h(v.surv_gid, v.survivors, np.uint32)
    want_start = gpsutil.d2h(v.surv_start, v.survivors, np.uint32)
    assert v.survivors > 100 and v.points > 0
    tiles = s.max_number_of_points // 256 + 2
    for call in range(2):
        gid = torch.full((n,), 0xFFFFFFFF, dtype=torch.int64, device="cuda").to(torch.int32)
        start = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        tfr = torch.full((tiles,), -1, dtype=torch.int32, device="cuda")
        ctr = torch.full((8,), -1, dtype=torch.int32, device="cuda")
        st = lib.gps_workload_scan_noalloc(ctypes.c_void_p(v.counts), ctypes.c_void_p(v.mask_last), n,
                                           s.max_number_of_points, ctypes.c_void_p(gid.data_ptr()),
                                           ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(tfr.data_ptr()),
                                           ctypes.c_void_p(ctr.data_ptr()), None)
        assert st == 0, lib.gps_last_error().decode()
        torch.cuda.synchronize()
        c = ctr.cpu().numpy().view(np.uint32)
        assert c[0] == v.survivors, f"call {call}: survivors {c[0]} vs {v.survivors}"
        assert c[2] == v.points, f"call {call}: points {c[2]} vs {v.points}"
        assert c[4] == 0
        got_gid = gid.cpu().numpy().view(np.uint32)[: v.survivors]
        got_start = start.cpu().numpy().view(np.uint32)[: v.survivors]
        assert np.array_equal(got_gid, want_gid), f"call {call}: survivor ids differ"
        assert np.array_equal(got_start, want_start), f"call {call}: first points differ"
        # every 256-point tile below P starts at the survivor owning its first point
        t = np.arange((int(v.points) + 255) // 256, dtype=np.int64) * 256
        owner = np.searchsorted(want_start.astype(np.int64), t, side="right") - 1
        assert np.array_equal(tfr.cpu().numpy().view(np.uint32)[: t.size], owner.astype(np.uint32))
    r.close()
    scene.close()


def test_noalloc_scan_rejects_oversized_input():
    lib = gpsplat.load_library()
    # null buffers: the size check answers first, and the null check would stop the call
    # before any device work if it did not
    for n in (0xFFFFFFFF, 65536 * 4096 + 1):
        st = lib.gps_workload_scan_noalloc(None, None, n, 100, None, None, None, None, None)
        assert st == 6, lib.gps_last_error()
        assert b"exceed" in lib.gps_last_error()
    st = lib.gps_workload_scan_noalloc(None, None, 4096, 100, None, None, None, None, None)
    assert st == 1
