"""Seeded synthetic 3DGS scenes and camera paths (stand-ins for the reference's evaluation
scenes, which are not distributed with it).

Scenes are produced as *raw* 3DGS PLY fields — pre-sigmoid opacity logits, log-scales,
un-normalised rot_0..rot_3 = (w, x, y, z), f_dc and channel-major f_rest — exactly what a
3DGS training run writes, so that both this library's loader and the reference's loader see
the same bytes.  `activate` turns raw fields into the CPUGaussian layout (mean, sh[48],
opacity, scale, rotation) for direct host upload.

  cube   : N Gaussians, positions U[-10,10]^3, log-scales N(-3,0.5), uniform random unit
           quaternions, opacity logit N(0,1.5), DC U[0,1], f_rest 0 (SH degree 0)
  town   : a 200x200 ground plane plus 400 axis-aligned boxes (footprint U[2,10]^2,
           height U[3,40]); Gaussians spread over the visible surfaces proportionally to
           area, flat along the surface normal (thin log N(-6,0.3), in-plane log N(-3,0.5)),
           random in-plane rotation, opacity logit N(2,1), DC U[0,1], 45 rest N(0,0.2);
           stored in 3D Morton order with the `bvh_sorted_order` comment so that every
           implementation keeps the file order
"""
from __future__ import annotations

import json

import numpy as np

RAW_FIELDS = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(45)] + [
    "opacity",
    "scale_0",
    "scale_1",
    "scale_2",
    "rot_0",
    "rot_1",
    "rot_2",
    "rot_3",
]


class RawScene:
    """Raw 3DGS fields: float32 arrays keyed like the PLY properties."""

    def __init__(self, pos, dc, rest, logit, log_scale, rot, sorted_order=False):
        self.pos = np.ascontiguousarray(pos, np.float32)
        self.dc = np.ascontiguousarray(dc, np.float32)
        self.rest = None if rest is None else np.ascontiguousarray(rest, np.float32)  # (N, 45) channel-major
        self.logit = np.ascontiguousarray(logit, np.float32)
        self.log_scale = np.ascontiguousarray(log_scale, np.float32)
        self.rot = np.ascontiguousarray(rot, np.float32)  # (N, 4) w, x, y, z
        self.sorted_order = sorted_order

    @property
    def n(self):
        return self.pos.shape[0]

    def subset(self, idx):
        return RawScene(self.pos[idx], self.dc[idx], None if self.rest is None else self.rest[idx], self.logit[idx],
                        self.log_scale[idx], self.rot[idx], self.sorted_order)

    def write_ply(self, path: str):
        n = self.n
        names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
        cols = [self.pos[:, 0], self.pos[:, 1], self.pos[:, 2], np.zeros(n, np.float32), np.zeros(n, np.float32),
                np.zeros(n, np.float32), self.dc[:, 0], self.dc[:, 1], self.dc[:, 2]]
        if self.rest is not None:
            names += [f"f_rest_{i}" for i in range(45)]
            cols += [self.rest[:, i] for i in range(45)]
        names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
        cols += [self.logit, self.log_scale[:, 0], self.log_scale[:, 1], self.log_scale[:, 2], self.rot[:, 0],
                 self.rot[:, 1], self.rot[:, 2], self.rot[:, 3]]
        rec = np.empty((n, len(names)), np.float32)
        for i, c in enumerate(cols):
            rec[:, i] = c
        header = ["ply", "format binary_little_endian 1.0"]
        if self.sorted_order:
            header.append("comment bvh_sorted_order")
        header.append(f"element vertex {n}")
        header += [f"property float {nm}" for nm in names]
        header.append("end_header")
        with open(path, "wb") as f:
            f.write(("\n".join(header) + "\n").encode())
            f.write(rec.tobytes())


def activate(raw: RawScene) -> np.ndarray:
    """CPUGaussian layout (59 float32 per Gaussian), activated in float32 like the loader."""
    n = raw.n
    out = np.zeros((n, 59), np.float32)
    out[:, 0:3] = raw.pos
    out[:, 3:6] = raw.dc
    if raw.rest is not None:
        for j in range(1, 16):
            for c in range(3):
                out[:, 3 + 3 * j + c] = raw.rest[:, (j - 1) + 15 * c]
    with np.errstate(over="ignore"):
        op = (np.float32(1.0) / (np.float32(1.0) + np.exp(-raw.logit))).astype(np.float32)
    out[:, 51] = np.clip(op, 0.0, 1.0)
    out[:, 52:55] = np.exp(raw.log_scale).astype(np.float32)
    q = raw.rot.astype(np.float32)
    d = (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + (q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3])
    out[:, 55:59] = q * (np.float32(1.0) / np.sqrt(d))[:, None]
    return out


def _uniform_quaternions(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


def cube(n: int, seed: int = 0x6A55) -> RawScene:
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-10.0, 10.0, (n, 3)).astype(np.float32)
    log_scale = rng.normal(-3.0, 0.5, (n, 3)).astype(np.float32)
    rot = _uniform_quaternions(rng, n)
    logit = rng.normal(0.0, 1.5, n).astype(np.float32)
    dc = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    return RawScene(pos, dc, None, logit, log_scale, rot)


def _rotmat_to_quat_wxyz(r: np.ndarray) -> np.ndarray:
    """Rotation matrices (N,3,3) with columns = local axes -> unit quaternions (w,x,y,z)."""
    m = r
    m00, m11, m22 = m[:, 0, 0], m[:, 1, 1], m[:, 2, 2]
    t = m00 + m11 + m22
    q = np.zeros((m.shape[0], 4))
    c0 = t > 0
    c1 = ~c0 & (m00 > m11) & (m00 > m22)
    c2 = ~c0 & ~c1 & (m11 > m22)
    c3 = ~c0 & ~c1 & ~c2
    s = np.sqrt(np.maximum(t + 1.0, 1e-12)) * 2
    q[c0] = np.stack([0.25 * s, (m[:, 2, 1] - m[:, 1, 2]) / s, (m[:, 0, 2] - m[:, 2, 0]) / s, (m[:, 1, 0] - m[:, 0, 1]) / s], 1)[c0]
    s = np.sqrt(np.maximum(1.0 + m00 - m11 - m22, 1e-12)) * 2
    q[c1] = np.stack([(m[:, 2, 1] - m[:, 1, 2]) / s, 0.25 * s, (m[:, 0, 1] + m[:, 1, 0]) / s, (m[:, 0, 2] + m[:, 2, 0]) / s], 1)[c1]
    s = np.sqrt(np.maximum(1.0 + m11 - m00 - m22, 1e-12)) * 2
    q[c2] = np.stack([(m[:, 0, 2] - m[:, 2, 0]) / s, (m[:, 0, 1] + m[:, 1, 0]) / s, 0.25 * s, (m[:, 1, 2] + m[:, 2, 1]) / s], 1)[c2]
    s = np.sqrt(np.maximum(1.0 + m22 - m00 - m11, 1e-12)) * 2
    q[c3] = np.stack([(m[:, 1, 0] - m[:, 0, 1]) / s, (m[:, 0, 2] + m[:, 2, 0]) / s, (m[:, 1, 2] + m[:, 2, 1]) / s, 0.25 * s], 1)[c3]
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


def morton_order(pos: np.ndarray) -> np.ndarray:
    mn = pos.min(axis=0)
    ext = np.maximum(pos.max(axis=0) - mn, 1e-9)
    g = np.clip(((pos - mn) / ext * 1023.0).astype(np.int64), 0, 1023)

    def spread(v):
        v = v.astype(np.uint64)
        out = np.zeros_like(v)
        for b in range(10):
            out |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b)
        return out

    code = spread(g[:, 0]) | (spread(g[:, 1]) << np.uint64(1)) | (spread(g[:, 2]) << np.uint64(2))
    return np.argsort(code, kind="stable")


TOWN_EXTENT = 200.0


def town_boxes(seed: int = 0x70A1, count: int = 400):
    rng = np.random.default_rng(seed ^ 0xB0B0)
    foot = rng.uniform(2.0, 10.0, (count, 2))
    height = rng.uniform(3.0, 40.0, count)
    centre = rng.uniform(-TOWN_EXTENT / 2 + 10, TOWN_EXTENT / 2 - 10, (count, 2))
    return foot, height, centre


def town(n: int, seed: int = 0x70A1, sh_degree: int = 3) -> RawScene:
    rng = np.random.default_rng(seed)
    foot, height, centre = town_boxes(seed)
    half = TOWN_EXTENT / 2
    # surfaces: ground (y=0), and per box: +x, -x, +z, -z sides, top
    faces = [("ground", None, TOWN_EXTENT * TOWN_EXTENT)]
    for b in range(len(height)):
        w, d = foot[b]
        h = height[b]
        faces += [("px", b, d * h), ("nx", b, d * h), ("pz", b, w * h), ("nz", b, w * h), ("top", b, w * d)]
    areas = np.array([f[2] for f in faces])
    fid = rng.choice(len(faces), size=n, p=areas / areas.sum())
    u = rng.uniform(0.0, 1.0, (n, 2))
    pos = np.zeros((n, 3))
    nrm = np.zeros((n, 3))
    tan = np.zeros((n, 3))
    kinds = np.array([f[0] for f in faces])
    boxes = np.array([-1 if f[1] is None else f[1] for f in faces])
    k = kinds[fid]
    bi = boxes[fid]
    g = k == "ground"
    pos[g, 0] = -half + u[g, 0] * TOWN_EXTENT
    pos[g, 2] = -half + u[g, 1] * TOWN_EXTENT
    nrm[g] = [0, 1, 0]
    tan[g] = [1, 0, 0]
    for kind, axis, sign in [("px", 0, 1), ("nx", 0, -1), ("pz", 2, 1), ("nz", 2, -1)]:
        sel = k == kind
        b = bi[sel]
        w, d, h = foot[b, 0], foot[b, 1], height[b]
        cx, cz = centre[b, 0], centre[b, 1]
        if axis == 0:
            pos[sel, 0] = cx + sign * w / 2
            pos[sel, 2] = cz - d / 2 + u[sel, 0] * d
            tan[sel] = [0, 0, 1]
        else:
            pos[sel, 2] = cz + sign * d / 2
            pos[sel, 0] = cx - w / 2 + u[sel, 0] * w
            tan[sel] = [1, 0, 0]
        pos[sel, 1] = u[sel, 1] * h
        nv = np.zeros(3)
        nv[axis] = sign
        nrm[sel] = nv
    sel = k == "top"
    b = bi[sel]
    pos[sel, 0] = centre[b, 0] - foot[b, 0] / 2 + u[sel, 0] * foot[b, 0]
    pos[sel, 2] = centre[b, 1] - foot[b, 1] / 2 + u[sel, 1] * foot[b, 1]
    pos[sel, 1] = height[b]
    nrm[sel] = [0, 1, 0]
    tan[sel] = [1, 0, 0]
    # random in-plane rotation of the tangent frame; local axes (t1, t2, n) carry scales (s0, s1, thin)
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    bit = np.cross(nrm, tan)
    t1 = np.cos(theta)[:, None] * tan + np.sin(theta)[:, None] * bit
    t2 = np.cross(nrm, t1)
    rmat = np.stack([t1, t2, nrm], axis=2)  # columns
    rot = _rotmat_to_quat_wxyz(rmat)
    log_scale = np.empty((n, 3), np.float32)
    log_scale[:, 0:2] = rng.normal(-3.0, 0.5, (n, 2))
    log_scale[:, 2] = rng.normal(-6.0, 0.3, n)
    logit = rng.normal(2.0, 1.0, n).astype(np.float32)
    dc = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    rest = rng.normal(0.0, 0.2, (n, 45)).astype(np.float32) if sh_degree > 0 else None
    order = morton_order(pos)
    raw = RawScene(pos[order], dc[order], None if rest is None else rest[order], logit[order], log_scale[order],
                   rot[order], sorted_order=True)
    return raw


def tile_town(raw: RawScene, copies_x: int, copies_z: int) -> RawScene:
    """GaussianEditor::Repeat-style tiling (translated copies of the whole scene)."""
    parts = []
    for i in range(copies_x):
        for j in range(copies_z):
            off = np.array([i * TOWN_EXTENT, 0.0, j * TOWN_EXTENT], np.float32)
            parts.append(off)
    n = raw.n
    pos = np.concatenate([raw.pos + o for o in parts])
    rep = len(parts)
    return RawScene(pos, np.tile(raw.dc, (rep, 1)), None if raw.rest is None else np.tile(raw.rest, (rep, 1)),
                    np.tile(raw.logit, rep), np.tile(raw.log_scale, (rep, 1)), np.tile(raw.rot, (rep, 1)),
                    sorted_order=raw.sorted_order)


# ---------------------------------------------------------------------------------
# camera paths
# ---------------------------------------------------------------------------------
def look_at_c2w(position, target, up=(0.0, 1.0, 0.0)):
    """3DGS camera-to-world rotation (columns right, down, forward) as a (3,3) matrix."""
    p = np.asarray(position, np.float64)
    f = np.asarray(target, np.float64) - p
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return np.stack([r, -u, f], axis=1)


def orbit(frames: int = 120, radius: float = 30.0, height: float = 10.0, target=(0.0, 0.0, 0.0)):
    out = []
    for i in range(frames):
        a = 2.0 * np.pi * i / frames
        p = np.array([radius * np.cos(a), height, radius * np.sin(a)])
        out.append((p, look_at_c2w(p, target)))
    return out


def random_poses(count: int, seed: int = 1):
    rng = np.random.default_rng(seed)
    out = []
    half = TOWN_EXTENT / 2
    for _ in range(count):
        p = np.array([rng.uniform(-half * 0.8, half * 0.8), rng.uniform(2.0, 30.0), rng.uniform(-half * 0.8, half * 0.8)])
        a = rng.uniform(0, 2 * np.pi)
        tgt = p + np.array([np.cos(a) * 20.0, -rng.uniform(1.0, 8.0), np.sin(a) * 20.0])
        out.append((p, look_at_c2w(p, tgt)))
    return out


def write_cameras_json(path: str, poses, width: int, height: int, fy: float, fx: float | None = None):
    cams = []
    for i, (p, r) in enumerate(poses):
        cams.append({
            "id": i,
            "img_name": f"frame_{i:04d}",
            "width": int(width),
            "height": int(height),
            "position": [float(v) for v in p],
            "rotation": [[float(v) for v in row] for row in np.asarray(r)],
            "fy": float(fy),
            "fx": float(fx if fx is not None else fy),
        })
    with open(path, "w") as f:
        json.dump(cams, f, indent=2)
