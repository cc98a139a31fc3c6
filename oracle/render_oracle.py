"""CPU restatement of the headless density renderer -- test infrastructure (the
oracle), not part of the product.

It follows the reference's visualiser, misc/volume_rendering_kernel.cu
(intersectBox :55-76, sample_tex / sample_tex_int :145-164, the DDA
get_next_hit :214-270, trace :272-318, render_surface :340-385, render_volume
:387-437) and the volume built by misc/volume_renderer.cpp:410-480, in float32
numpy arithmetic (no fused multiply-adds, like the library's renderer, which is
compiled without them), with the library's deliberate differences: random
numbers from the PCG hash (Jarzynski & Olano 2020) keyed by pixel, frame and
draw; the primary direction normalised by division; point sampling of voxel
clamp(floor(t * res)).  cos, sin and exp come from numpy's float32 functions,
which may differ from CUDA's in the last bits, so images agree up to rare
pixels.

Parity unpinned: the reference renders through OpenGL and a window, which this
machine cannot run; the restatement is checked against the GPU renderer.
"""
from __future__ import annotations

import numpy as np

F = np.float32
MAX_STEPS = 1025
TSTEP = F(0.01)


def pcg_hash(v):
    v = np.asarray(v, np.uint32)
    state = v * np.uint32(747796405) + np.uint32(2891336453)
    word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


class Rng:
    def __init__(self, npix: int, frame: int, seed: int):
        pix = np.arange(npix, dtype=np.uint32)
        with np.errstate(over="ignore"):
            inner = pcg_hash(np.uint32((seed + frame * 0x9E3779B9) & 0xFFFFFFFF))
            self.key = pcg_hash(pix + inner)
        self.n = 0

    def next(self, sel=None):
        with np.errstate(over="ignore"):
            h = pcg_hash(self.key + np.uint32(self.n))
        self.n += 1
        r = ((h >> np.uint32(8)) + np.uint32(1)).astype(F) * F(1.0 / 16777216.0)
        return r if sel is None else r[sel]


def build_volume(base, density, reverse_mapping: bool = False):
    """(voxels uint8 [D][H][W] as x fastest, res (W, H, D)) of the cells with
    positive density (volume_renderer.cpp:410-480)."""
    base = np.asarray(base, np.int64).reshape(-1, 3)
    d = np.asarray(density, np.float64).reshape(-1, 64)
    e = np.arange(64)
    loc = np.stack([e >> 4, (e >> 2) & 3, e & 3], 1)
    cells = base[:, None, :] + loc[None]
    pos = d > 0
    lo = cells[pos].min(axis=0)
    hi = cells[pos].max(axis=0) + 1
    res = hi - lo
    vox = np.zeros((res[2], res[1], res[0]), np.uint8)
    c = cells.reshape(-1, 3) - lo
    v = d.reshape(-1).copy()
    if reverse_mapping:
        m = v > 0
        v[m] = np.power(v[m] - 1e-6, 0.33333333) * (1 - 1e-6)
    q = np.where(v != 0, np.clip((v * 254).astype(np.int64), 0, 254) + 1, 0).astype(np.uint8)
    ok = ((c >= 0) & (c < res)).all(axis=1)
    vox[c[ok, 2], c[ok, 1], c[ok, 0]] = q[ok]
    return vox, res


class Volume:
    def __init__(self, vox, res, slice_=0.99999, mirror=""):
        self.vox = vox
        self.res = np.asarray(res)
        rmax = F(int(self.res.max()))
        self.scale = np.array([F(2) if a in mirror else F(1) for a in "xyz"], F)
        self.box_size = np.array([F(int(r)) / rmax * s for r, s in zip(self.res, self.scale)], F)
        self.box_res = np.array([F(int(r)) * s for r, s in zip(self.res, self.scale)], F)
        self.tex_res = np.array([F(int(r)) for r in self.res], F)   # the texture keeps the volume's size
        self.slice = F(slice_)

    def point_sample(self, p):
        # wrap_coord (:133-143): box_scale 2 on mirrored axes reflects past the far face
        p = (p * F(0.5) + F(0.5)) * self.scale
        p = np.where(p > 1, F(2) - p, p)
        p = p * F(2) + F(-1.0)
        t = p * F(0.5) + F(0.5)
        i = np.floor(t * self.tex_res).astype(np.int64)
        i = np.clip(i, 0, self.res - 1)
        return self.vox[i[:, 2], i[:, 1], i[:, 0]].astype(F) / F(255.0)

    def _gate(self, p):
        inside = np.all((F(-1.0) < p) & (p < F(1.0)), axis=1)
        return inside & ~(p[:, 2] > F(2) * self.slice - F(1))

    def sample_world(self, pos):
        p = pos / self.box_size
        ok = self._gate(p)
        out = np.zeros(len(p), F)
        if ok.any():
            out[ok] = self.point_sample(p[ok])
        return out

    def sample_voxel(self, ipos):
        p = ((ipos + F(0.5)) / self.box_res) * F(2) + F(-1.0)
        ok = self._gate(p)
        out = np.zeros(len(p), F)
        if ok.any():
            out[ok] = self.point_sample(p[ok])
        return out


def intersect_box(o, d, bmin, bmax):
    inv = F(1.0) / d
    tbot = inv * (bmin - o)
    ttop = inv * (bmax - o)
    tmin = np.fmin(ttop, tbot)
    tmax = np.fmax(ttop, tbot)
    tnear = np.fmax(np.fmax(tmin[:, 0], tmin[:, 1]), np.fmax(tmin[:, 0], tmin[:, 2]))
    tfar = np.fmin(np.fmin(tmax[:, 0], tmax[:, 1]), np.fmin(tmax[:, 0], tmax[:, 2]))
    return tfar > tnear, tnear


def next_hit(V: Volume, o, d, threshold):
    """DDA get_next_hit for every ray: (hit bool[n], hit position [n][3])."""
    n = len(o)
    ln = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    d = d / ln[:, None]
    box, tnear = intersect_box(o, d, -V.box_size, V.box_size)
    tnear = np.where(tnear < F(0), F(0), tnear)
    pos = o + d * (tnear + F(1e-4))[:, None]
    ri = F(1.0) / d
    rs = np.where(d > 0, F(1), np.where(d < 0, F(-1), F(0))).astype(F)
    org = ((pos + V.box_size) * F(0.5)) * (V.box_res[0] / V.box_size[0])
    ipos = np.floor(org)
    dis = (((ipos - org) + F(0.5)) + rs * F(0.5)) * ri
    ratio = V.box_size[0] / V.box_res[0]
    hit = np.zeros(n, bool)
    hit_pos = np.zeros((n, 3), F)
    active = box.copy()
    thr = F(threshold)
    for _ in range(MAX_STEPS):
        idx = np.nonzero(active)[0]
        if len(idx) == 0:
            break
        s = V.sample_voxel(ipos[idx])
        h = s > thr
        if h.any():
            k = idx[h]
            mini = (((ipos[k] - org[k]) + F(0.5)) - rs[k] * F(0.5)) * ri[k]
            t = np.fmax(mini[:, 0], np.fmax(mini[:, 1], mini[:, 2])) * ratio * F(2.0)
            hit_pos[k] = pos[k] + d[k] * t[:, None]
            hit[k] = True
            active[k] = False
        k = idx[~h]
        dk = dis[k]
        mx = (dk[:, 0] <= dk[:, 1]) & (dk[:, 0] < dk[:, 2])
        my = ~mx & (dk[:, 1] <= dk[:, 0]) & (dk[:, 1] <= dk[:, 2])
        mz = ~mx & ~my
        mm = np.stack([mx, my, mz], 1).astype(F)
        dis[k] = dk + (mm * rs[k]) * ri[k]
        ipos[k] = ipos[k] + mm * rs[k]
    return hit, hit_pos


def camera_rays(camera, W, H, r0, r1):
    C = np.asarray(camera, F).reshape(3, 4)
    y, x = np.divmod(np.arange(W * H), W)
    u = ((x.astype(F) + r0) / F(W)) * F(2.0) - F(1.0)
    v = ((y.astype(F) + r1) / F(W)) * F(2.0) - F(1.0)
    o = np.broadcast_to(C[:, 3], (W * H, 3)).astype(F)
    dirv = np.stack([u, v, np.full_like(u, F(-2.0))], 1)
    ln = np.sqrt(dirv[:, 0] * dirv[:, 0] + dirv[:, 1] * dirv[:, 1] + dirv[:, 2] * dirv[:, 2])
    dirv = dirv / ln[:, None]
    d = np.stack([dirv[:, 0] * C[r, 0] + dirv[:, 1] * C[r, 1] + dirv[:, 2] * C[r, 2] for r in range(3)], 1)
    return u, v, o, d


def pack_rgba(r, g, b, a):
    def q(x):
        return (np.clip(x, F(0), F(1)) * F(255)).astype(np.uint32)
    return (q(a) << np.uint32(24)) | (q(b) << np.uint32(16)) | (q(g) << np.uint32(8)) | q(r)


def render(base, density, width, height, camera, mode=0, frames=1, threshold=0.5, extinction=1.0,
           slice_=0.99999, seed=0, reverse_mapping=False, mirror=""):
    """The image as uint32 [height][width] (a<<24 | b<<16 | g<<8 | r), row 0 at the bottom."""
    vox, res = build_volume(base, density, reverse_mapping)
    V = Volume(vox, res, slice_, mirror)
    npix = width * height
    buf = np.zeros((npix, 3), F)
    out = None
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for f in range(1, frames + 1):
            rng = Rng(npix, f, seed)
            r0, r1 = rng.next(), rng.next()
            u, v, o, d = camera_rays(camera, width, height, r0, r1)
            if mode == 0:
                col = np.tile(np.array([0.86, 0.85, 0.9], F), (npix, 1))
                hit, pos = next_hit(V, o, d, threshold)
                hp = np.nonzero(hit)[0]
                col[hp] = 0
                for _ in range(3):
                    a, b = rng.next(hp), rng.next(hp)
                    sx = a * F(2) - F(1)
                    phi = b * F(2) * F(3.14159265358979)
                    yz = np.sqrt(F(1) - sx * sx)
                    dirv = np.stack([sx, yz * np.cos(phi), yz * np.sin(phi)], 1).astype(F)
                    blocked, _ = next_hit(V, pos[hp], dirv, threshold)
                    dt = dirv[:, 0] * F(0.6) + dirv[:, 1] * F(0.75) + dirv[:, 2] * F(0.15)
                    c1 = np.fmax(F(0), np.fmin(dt * F(0.5) + F(0.5), F(1)))
                    light = np.array([0.9, 0.7, 0.3], F)[None] * c1[:, None] + \
                        np.array([0.4, 0.5, 0.9], F)[None] * (F(1) - c1)[:, None]
                    add = light * (F(2.0) / F(3))
                    col[hp] = np.where(blocked[:, None], col[hp], col[hp] + add)
            else:
                s = np.zeros(npix, F)
                box, tnear = intersect_box(o, d, -V.box_size, V.box_size)
                tnear = np.where(tnear < F(0), F(0), tnear)
                pos = o + d * (tnear + F(1e-4))[:, None]
                step = d * TSTEP
                for _ in range(MAX_STEPS):
                    r = rng.next()
                    smp = V.sample_world(pos + step * r[:, None])
                    s = np.where(box, s + smp, s)
                    pos = pos + step
                s = (s.astype(np.float64) * 1e-2).astype(F)
                s = np.fmax(s - F(threshold) * F(1), F(0))
                e = F(1) - np.exp(-F(extinction) * s)
                g = F(1) - e
                col = np.stack([g, g, g], 1)
            buf += col
            if f == frames:
                sc = F(1.0) - F(0.15) * (u * u + v * v)
                n = F(f)
                out = pack_rgba(sc * (buf[:, 0] / n), sc * (buf[:, 1] / n), sc * (buf[:, 2] / n), sc * F(1.0))
    return out.reshape(height, width), res

