"""Seeded synthetic RGB-D frame pairs with analytic 3-D ground-truth motion.

The reference ships no dataset; these scenes stand in for its Kinect PNG pairs:
  * a random-texture background plane at z = 3 m and N textured planar patches
    (random pose, centre depth in [0.8, 2.5] m) seen by a pinhole camera (f, cx, cy);
  * frame 2 moves every patch by its own rigid motion (rotation <= 3 deg about a random axis
    through the patch centre, translation <= 3 cm); the background stays;
  * colour is uint8 BGR from a texture attached to each surface (brightness constancy holds),
    plus Gaussian colour noise (sigma 2 of 255);
  * depth is metres with noise N(0, (1.45e-3 z^2)^2), quantised to millimetres (the uint16-mm
    PNG the demo reads, src/main.cpp:32-43), with a fraction of zero (invalid) pixels made of
    small blobs and isolated dropouts.
Ground truth is the per-pixel motion of frame 1's surface point: u, v in pixels, w in metres.

3-D endpoint error (the reference has none; this definition is the build's):
  P1 = z K^-1 (x, y, 1),  P2 = (z + w) K^-1 (x + u, y + v, 1),  EPE = |(P2 - P1) - (P2* - P1*)|
over pixels where frame-1 depth is valid, with z the true frame-1 depth.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class Camera:
    f: float
    cx: float
    cy: float


# Named workloads with their generator settings.
CONFIGS = {
    "320x240": dict(W=320, H=240, f=262.5, cx=159.5, cy=119.5, n_patches=3, hole_frac=0.05),
    "640x480": dict(W=640, H=480, f=525.0, cx=319.5, cy=239.5, n_patches=6, hole_frac=0.08),
    "160x120": dict(W=160, H=120, f=131.25, cx=79.5, cy=59.5, n_patches=3, hole_frac=0.05),
}


def _rotation(axis, angle):
    axis = axis / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * (K @ K)


class _Texture:
    """Multi-octave value noise over local surface coordinates (s, t) in metres -> BGR 0..255."""

    def __init__(self, rng, s_range, t_range, cells=(0.04, 0.015, 0.006)):
        self.s0, self.s1 = s_range
        self.t0, self.t1 = t_range
        self.octaves = []
        amp = [0.55, 0.3, 0.15]
        for c, a in zip(cells, amp):
            gw = int(np.ceil((self.s1 - self.s0) / c)) + 2
            gh = int(np.ceil((self.t1 - self.t0) / c)) + 2
            self.octaves.append((c, a, rng.random((gh, gw, 3))))
        self.base = rng.uniform(0.2, 0.8, 3)
        self.contrast = rng.uniform(0.6, 1.0)

    def __call__(self, s, t):
        out = np.zeros(s.shape + (3,))
        for c, a, g in self.octaves:
            x = np.clip((s - self.s0) / c, 0, g.shape[1] - 1.001)
            y = np.clip((t - self.t0) / c, 0, g.shape[0] - 1.001)
            x0 = np.floor(x).astype(np.int64)
            y0 = np.floor(y).astype(np.int64)
            fx = (x - x0)[..., None]
            fy = (y - y0)[..., None]
            v = (g[y0, x0] * (1 - fx) * (1 - fy) + g[y0, x0 + 1] * fx * (1 - fy) +
                 g[y0 + 1, x0] * (1 - fx) * fy + g[y0 + 1, x0 + 1] * fx * fy)
            out += a * (v - 0.5)
        col = self.base + self.contrast * out
        return np.clip(col, 0, 1) * 255.0


class _Patch:
    def __init__(self, rng, cam, W, H):
        z = rng.uniform(0.8, 2.5)
        px = rng.uniform(0.15 * W, 0.85 * W)
        py = rng.uniform(0.15 * H, 0.85 * H)
        self.c = np.array([(px - cam.cx) * z / cam.f, (py - cam.cy) * z / cam.f, z])
        tilt = _rotation(rng.normal(size=3) * np.array([1, 1, 0.2]), np.deg2rad(rng.uniform(0, 35)))
        self.a1 = tilt @ np.array([1.0, 0, 0])
        self.a2 = tilt @ np.array([0, 1.0, 0])
        self.half = np.array([rng.uniform(0.10, 0.25), rng.uniform(0.10, 0.25)]) * z
        self.tex = _Texture(rng, (-self.half[0], self.half[0]), (-self.half[1], self.half[1]))
        ang = np.deg2rad(rng.uniform(0, 3.0))
        self.R = _rotation(rng.normal(size=3), ang)
        d = rng.normal(size=3)
        self.T = d / np.linalg.norm(d) * rng.uniform(0, 0.03)

    def moved(self):
        q = _Patch.__new__(_Patch)
        q.c = self.c + self.T
        q.a1 = self.R @ self.a1
        q.a2 = self.R @ self.a2
        q.half = self.half
        q.tex = self.tex
        q.R, q.T = self.R, self.T
        return q


def _render(cam, W, H, patches, bg_tex, bg_z=3.0):
    xs, ys = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    d = np.stack([(xs - cam.cx) / cam.f, (ys - cam.cy) / cam.f, np.ones_like(xs)], -1)
    zbuf = np.full((H, W), bg_z)
    sid = np.full((H, W), -1, np.int64)
    st = np.stack([d[..., 0] * bg_z, d[..., 1] * bg_z], -1)
    for k, p in enumerate(patches):
        n = np.cross(p.a1, p.a2)
        den = d @ n
        with np.errstate(divide="ignore", invalid="ignore"):
            lam = (n @ p.c) / den
        P = d * lam[..., None]
        rel = P - p.c
        s = rel @ p.a1
        t = rel @ p.a2
        hit = (lam > 0.05) & (np.abs(s) <= p.half[0]) & (np.abs(t) <= p.half[1]) & (lam < zbuf)
        zbuf = np.where(hit, lam, zbuf)
        sid = np.where(hit, k, sid)
        st = np.where(hit[..., None], np.stack([s, t], -1), st)
    col = np.zeros((H, W, 3))
    bgm = sid < 0
    col[bgm] = bg_tex(st[bgm][:, 0], st[bgm][:, 1])
    for k, p in enumerate(patches):
        m = sid == k
        if m.any():
            col[m] = p.tex(st[m][:, 0], st[m][:, 1])
    return col, zbuf, sid, d


def _holes(rng, H, W, frac):
    mask = np.zeros((H, W), bool)
    target = int(frac * H * W)
    blob_budget = int(0.6 * target)
    yy, xx = np.mgrid[-4:5, -4:5]
    while mask.sum() < blob_budget:
        r = rng.uniform(1.0, 4.0)
        cy, cx = rng.integers(0, H), rng.integers(0, W)
        m = (yy ** 2 + xx ** 2) <= r * r
        y0, x0 = cy - 4, cx - 4
        ys = slice(max(0, y0), min(H, y0 + 9))
        xs_ = slice(max(0, x0), min(W, x0 + 9))
        mask[ys, xs_] |= m[ys.start - y0:ys.stop - y0, xs_.start - x0:xs_.stop - x0]
    rest = max(0, target - int(mask.sum()))
    idx = rng.choice(H * W, size=rest, replace=False)
    mask.flat[idx] = True
    return mask


def _motion_gt(cam, W, H, patches, z1, sid1, d):
    """Analytic motion (u px, v px, w m) of the surface points seen in a frame when every patch
    makes its rigid motion; the background stays."""
    P1 = d * z1[..., None]
    P2 = P1.copy()
    for k, p in enumerate(patches):
        m = sid1 == k
        P2[m] = (P1[m] - p.c) @ p.R.T + p.c + p.T
    x2 = cam.f * P2[..., 0] / P2[..., 2] + cam.cx
    y2 = cam.f * P2[..., 1] / P2[..., 2] + cam.cy
    xs, ys = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    return np.stack([x2 - xs, y2 - ys, P2[..., 2] - z1], -1).astype(np.float32)


def make_pair(W=640, H=480, f=525.0, cx=319.5, cy=239.5, n_patches=6, hole_frac=0.08, seed=0,
              color_noise=2.0, depth_noise=1.45e-3):
    """One frame pair.  Returns a dict with bgr1, bgr2 (H,W,3 uint8), depth1, depth2 (H,W float32
    metres, 0 = invalid), gt (H,W,3 float32: u px, v px, w m), z1_true (H,W float64) and cam."""
    rng = np.random.default_rng(seed)
    cam = Camera(f, cx, cy)
    ext = 3.0 / f * max(W, H) + 0.5
    bg_tex = _Texture(rng, (-ext, ext), (-ext, ext), cells=(0.12, 0.05, 0.02))
    patches = [_Patch(rng, cam, W, H) for _ in range(n_patches)]
    moved = [p.moved() for p in patches]
    col1, z1, sid1, d = _render(cam, W, H, patches, bg_tex)
    col2, z2, _, _ = _render(cam, W, H, moved, bg_tex)
    gt = _motion_gt(cam, W, H, patches, z1, sid1, d)

    def sensor(col, z):
        c = np.clip(np.rint(col + rng.normal(0, color_noise, col.shape)), 0, 255).astype(np.uint8)
        zn = z + rng.normal(0, 1, z.shape) * depth_noise * z * z
        mm = np.clip(np.rint(zn * 1000.0), 0, 65535).astype(np.uint16)
        dep = (mm * 0.001).astype(np.float32)
        dep[_holes(rng, H, W, hole_frac)] = 0
        return c, dep

    bgr1, depth1 = sensor(col1, z1)
    bgr2, depth2 = sensor(col2, z2)
    return dict(bgr1=bgr1, depth1=depth1, bgr2=bgr2, depth2=depth2, gt=gt, z1_true=z1, cam=cam,
                W=W, H=H, seed=seed)


def make_sequence(W=640, H=480, f=525.0, cx=319.5, cy=239.5, n_patches=6, hole_frac=0.08, n_frames=16, seed=0,
                  color_noise=2.0, depth_noise=1.45e-3):
    """Frames of one camera stream: every patch follows a smooth rigid trajectory (a fixed per-frame
    rotation <= 3 deg about its centre and translation <= 3 cm, so frame t+1 relates to frame t like
    the two frames of make_pair).  Returns a list of dicts with bgr (H,W,3 uint8) and depth (H,W
    float32 m, 0 = invalid)."""
    rng = np.random.default_rng(seed)
    cam = Camera(f, cx, cy)
    ext = 3.0 / f * max(W, H) + 0.5
    bg_tex = _Texture(rng, (-ext, ext), (-ext, ext), cells=(0.12, 0.05, 0.02))
    patches = [_Patch(rng, cam, W, H) for _ in range(n_patches)]
    frames = []
    cur = patches
    for t in range(n_frames):
        col, z, sid, d = _render(cam, W, H, cur, bg_tex)
        c = np.clip(np.rint(col + rng.normal(0, color_noise, col.shape)), 0, 255).astype(np.uint8)
        zn = z + rng.normal(0, 1, z.shape) * depth_noise * z * z
        dep = (np.clip(np.rint(zn * 1000.0), 0, 65535).astype(np.uint16) * 0.001).astype(np.float32)
        dep[_holes(rng, H, W, hole_frac)] = 0
        # gt_next: the analytic motion of this frame's surface points to the next frame
        frames.append(dict(bgr=c, depth=dep, z_true=z, gt_next=_motion_gt(cam, W, H, cur, z, sid, d)))
        cur = [p.moved() for p in cur]
    return dict(frames=frames, cam=cam, W=W, H=H)


def make_config_pair(name, seed=0):
    c = dict(CONFIGS[name])
    return make_pair(seed=seed, **c)


def epe3d(flow, gt, z, cam, mask):
    """Mean and max 3-D endpoint error (metres) of flow (H,W,3) against gt (H,W,3) with depth z."""
    H, W = z.shape
    xs, ys = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))

    def disp(fl):
        fl = fl.astype(np.float64)
        x2, y2, z2 = xs + fl[..., 0], ys + fl[..., 1], z + fl[..., 2]
        P1 = np.stack([(xs - cam.cx) / cam.f * z, (ys - cam.cy) / cam.f * z, z], -1)
        P2 = np.stack([(x2 - cam.cx) / cam.f * z2, (y2 - cam.cy) / cam.f * z2, z2], -1)
        return P2 - P1

    e = np.linalg.norm(disp(flow) - disp(gt), axis=-1)[mask]
    if e.size == 0:
        return 0.0, 0.0
    return float(e.mean()), float(e.max())
