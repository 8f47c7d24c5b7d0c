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


def _expected_scan(counts, bits, max_points):
    """What the scan must produce, in numpy: survivors in Gaussian order, exclusive point
    offsets mod 2^32, P = min(total, max_points) and each 256-point tile's first survivor."""
    gid = np.nonzero(bits)[0].astype(np.uint32)
    c = counts[gid].astype(np.uint64)
    ex = np.concatenate([np.zeros(1, np.uint64), np.cumsum(c, dtype=np.uint64)[:-1]])
    start = (ex & np.uint64(0xFFFFFFFF)).astype(np.uint32) if gid.size else np.zeros(0, np.uint32)
    total = int(c.sum()) & 0xFFFFFFFF
    points = min(total, max_points)
    t = np.arange((points + 255) // 256, dtype=np.int64) * 256
    owner = (np.searchsorted(start.astype(np.int64), t, side="right") - 1).astype(np.uint32)
    return gid, start, total, points, int(total > max_points), owner


def _run_exact_size(lib, counts, bits, max_points):
    """Runs the scan on device buffers of exactly the documented sizes: counts up to n rounded
    up to a multiple of 4, ceil(n / 32) mask words (with junk bits past n in the last word)."""
    import torch

    n = counts.size
    c4 = np.zeros((n + 3) // 4 * 4, np.uint32)
    c4[:n] = counts
    words = np.zeros((n + 31) // 32 * 32, np.uint8)
    words[:n] = bits
    words[n:] = 1  # must be ignored
    mask = np.packbits(words, bitorder="little").view(np.uint32)
    d_counts = torch.from_numpy(c4.view(np.int32)).cuda()
    d_mask = torch.from_numpy(mask.view(np.int32)).cuda()
    gid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    start = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    tiles = max_points // 256 + 2
    tfr = torch.full((tiles,), -1, dtype=torch.int32, device="cuda")
    ctr = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    st = lib.gps_workload_scan_noalloc(ctypes.c_void_p(d_counts.data_ptr()), ctypes.c_void_p(d_mask.data_ptr()), n,
                                       max_points, ctypes.c_void_p(gid.data_ptr()), ctypes.c_void_p(start.data_ptr()),
                                       ctypes.c_void_p(tfr.data_ptr()), ctypes.c_void_p(ctr.data_ptr()), None)
    assert st == 0, lib.gps_last_error().decode()
    torch.cuda.synchronize()
    return (gid.cpu().numpy().view(np.uint32), start.cpu().numpy().view(np.uint32), tfr.cpu().numpy().view(np.uint32),
            ctr.cpu().numpy().view(np.uint32))


# odd sizes (partial last mask word, counts not a multiple of 16), and n = 2^25, the first size
# that takes the scan's four-round tiles, with and without truncation
@pytest.mark.parametrize("n,density,max_points", [(4097, 0.5, 10**6), (60001, 0.3, 10**6), (60001, 0.9, 50000),
                                                  (33554432, 0.3, 250_000_000), (33554432, 0.3, 40_000_000)])
def test_noalloc_scan_matches_numpy(n, density, max_points):
    lib = gpsplat.load_library()
    rng = np.random.default_rng(n ^ int(density * 100) ^ max_points)
    counts = rng.integers(0, 21, n, dtype=np.uint32)
    bits = rng.random(n) < density
    gid_w, start_w, total, points, trunc, owner_w = _expected_scan(counts, bits, max_points)
    for call in range(2):
        gid, start, tfr, c = _run_exact_size(lib, counts, bits, max_points)
        assert c[0] == gid_w.size and c[1] == total and c[2] == points and c[3] == trunc, f"call {call}: counters {c[:4]}"
        assert np.array_equal(gid[: gid_w.size], gid_w), f"call {call}: survivor ids differ"
        assert np.array_equal(start[: gid_w.size], start_w), f"call {call}: first points differ"
        assert np.array_equal(tfr[: owner_w.size], owner_w), f"call {call}: tile owners differ"


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
