"""The render path's workload scan on scenes of 32M Gaussians and more (scan tiles of 16,384
Gaussians, four rounds per thread: workload_distributor.cu:52-145 restated for large scenes).

The 60k town in the half format is tiled 560 times (33.6M Gaussians) and rendered with culling
and occlusion. The pass's compacted survivors must be the mask's set bits in Gaussian order,
their first points the exclusive prefix sum of their point counts (mod 2^32, as the
reference's u32 offsets), and the pass's point count the clamped total. The splat buffer must
not depend on the walk order: the screen-binned walk and the Gaussian-order walk (forced with
GPS_BIN_CROWDED=0) give the same buffer bit for bit.
"""
import numpy as np
import pytest

import gpsplat
import gpsutil
import synth

pytestmark = pytest.mark.gpu


def _tiled():
    ply = gpsutil.cached_ply("town60k", lambda: synth.town(60000, seed=5))
    base = gpsplat.Scene.from_ply(ply, gpsplat.GPS_SCENE_HALF)
    offs = [[(i - 13.5) * 220.0, (j - 9.5) * 220.0] for j in range(20) for i in range(28)]
    scene = base.tile(offs)
    base.close()
    assert scene.count == 560 * 60000 >= (32 << 20)
    return scene


def _frame(scene, s, monkeypatch=None, crowded=None):
    if crowded is not None:
        monkeypatch.setenv("GPS_BIN_CROWDED", crowded)
    r = gpsplat.Renderer(scene, s)
    loop = gpsplat.FrameLoop(r)
    cams = gpsutil.cameras_for(s, synth.orbit(2, 30.0, 10.0))
    for cam in cams:
        loop.step(cam)
    gpsutil.sync()
    n = scene.count
    v = r.debug_view()
    out = {
        "counts": gpsutil.d2h(v.counts, n, np.uint32),
        "mask": gpsutil.mask_bits(gpsutil.d2h(v.mask_last, (n + 31) // 32, np.uint32), n),
        "surv_gid": gpsutil.d2h(v.surv_gid, v.survivors, np.uint32),
        "surv_start": gpsutil.d2h(v.surv_start, v.survivors, np.uint32),
        "points": int(v.points),
        "buffer": gpsutil.d2h(*r.splat_buffer(), np.uint64),
        "stats": r.stats(),
    }
    loop.close()
    r.close()
    return out


def test_big_scene_scan_and_walk_order(monkeypatch):
    scene = _tiled()
    s = gpsplat.default_settings(width=1920, height=1080, supersampling_factor=2, samples_per_pixel=4)
    a = _frame(scene, s)
    gid = np.nonzero(a["mask"])[0].astype(np.uint32)
    assert gid.size > 100_000
    assert np.array_equal(a["surv_gid"], gid)
    cnt = a["counts"][gid].astype(np.uint64)
    assert (cnt > 0).all()
    first = (np.concatenate([[0], np.cumsum(cnt)[:-1]]) % (1 << 32)).astype(np.uint32)
    assert np.array_equal(a["surv_start"], first)
    assert a["points"] == min(int(cnt.sum()) % (1 << 32), s.max_number_of_points)
    st = a["stats"]
    assert st.screen_order_one == 1 or st.screen_order_two == 1, "no pass took the screen-binned walk"
    b = _frame(scene, s, monkeypatch, crowded="0")
    assert (b["stats"].screen_order_one, b["stats"].screen_order_two) == (0, 0)
    assert np.array_equal(a["mask"], b["mask"])
    assert np.array_equal(a["buffer"], b["buffer"])
    scene.close()
