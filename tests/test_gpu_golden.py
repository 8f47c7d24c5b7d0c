"""Bit-exact parity of the CUDA path against golden fixtures produced by the reference's own
kernels (tests/golden/make_golden.py ran the reference build on a B200 and stored what it
rendered).  Runs without the reference: scenes are regenerated from their seeds (the PLY bytes
are checked against the recorded hash) and rendered through the C-ABI frame loop."""
import glob
import hashlib
import os

import numpy as np
import pytest

import gpsplat
import gpsutil

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cases():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "case_*.npz")))


def _sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def _cams_from(rec):
    cams = []
    for r in rec:
        c = gpsplat.Camera()
        for k, n in (("view", 16), ("proj", 16), ("position", 3)):
            getattr(c, k)[:] = [float(v) for v in r[k]]
        c.frustum_planes[:] = [float(v) for v in r["planes"]]
        c.frame = int(r["frame"])
        c.camera_moved = int(r["camera_moved"])
        cams.append(c)
    return cams


@pytest.mark.parametrize("case", _cases())
def test_golden_bit_exact(case):
    import sys

    sys.path.insert(0, GOLDEN)
    import make_golden

    make, tag, overrides, poses, variant, fmt = make_golden.CASES[case]
    gold = np.load(os.path.join(GOLDEN, f"case_{case}.npz"))
    ply = gpsutil.cached_ply(tag, make)
    assert _sha(ply) == str(gold["ply_sha256"]), "synthetic scene generator drifted from the fixture"
    s = gpsplat.default_settings(**overrides)
    cams = _cams_from(gold["cameras"])
    scene = gpsplat.Scene.from_ply(ply, fmt)
    n = scene.count
    mine = gpsutil.run_mine(scene, s, cams)
    problems = []
    for f, m in enumerate(mine):
        pre = f"f{f}_"
        if not np.array_equal(gold[pre + "buffer"], m["buffer"]):
            problems.append(f"frame {f}: splat buffer differs at {np.count_nonzero(gold[pre + 'buffer'] != m['buffer'])} entries")
        for key in ("image", "depth", "hiz"):
            g = gold[pre + key]
            mk = m["image_pre_post"] if key == "image" else m[key]
            if not np.array_equal(g.view(np.uint32), mk.view(np.uint32)):
                problems.append(f"frame {f}: {key} differs at {np.count_nonzero(g != mk)} values")
        if not np.array_equal(gold[pre + "mask_last"], m["mask_last"]):
            problems.append(f"frame {f}: survivor mask differs")
        ml = gpsutil.mask_bits(m["mask_last"], n)
        if not np.array_equal(gpsutil.offsets_from(m["counts"], gpsutil.written_mask(m, n)), gold[pre + "offsets"]):
            problems.append(f"frame {f}: point offsets differ")
        ids = gold[pre + "color_ids"]
        if not np.array_equal(gold[pre + "colors"].view(np.uint32), m["colors_rec"][ids].view(np.uint32)):
            problems.append(f"frame {f}: SH colours differ")
        st = gold[pre + "stats"]
        if (m["stats_obj"].num_points_one, m["stats_obj"].num_points_two) != (int(st[0]), int(st[1])):
            problems.append(f"frame {f}: point counts differ")
    assert not problems, "\n".join(problems)
