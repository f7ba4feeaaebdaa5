"""FP64 autograd restatement of the colour2 VBD step -- TEST INFRASTRUCTURE ONLY.

A vectorised torch (float64) version of the same update the C++ oracle restates
(YarnBall/sim/iteration.cu:8-74, YarnBall/sim/cosserat.cu:112-161, 246-337,
SDFCollisionSolver/cudaSDFCollision.cu:88-155, 205-268), written so that torch.autograd can
differentiate a rollout.  It is the FP64 reference gradient for the solver's hand-written
adjoint, and is only used by tests.  Supported: colour2 schedule, wind (iteration.cu:18-30; the
clock starts at `time` and advances by dt per step), any substep count, SDF pass with a
rotated/translated body.  The sign tests of the orientation update and the SDF
branch are treated as constants (their derivative is zero almost everywhere).
"""
from __future__ import annotations

import numpy as np
import torch

HAS_PREV, HAS_NEXT, HAS_NEXT_ORIENTATION, FIX_ORIENTATION = 1, 2, 4, 8


def qmul(l, r):
    lx, ly, lz, lw = l.unbind(-1)
    rx, ry, rz, rw = r.unbind(-1)
    return torch.stack([lw * rx + rw * lx + (ly * rz - ry * lz), lw * ry + rw * ly + (lz * rx - rz * lx),
                        lw * rz + rw * lz + (lx * ry - rx * ly), lw * rw - (lx * rx + ly * ry + lz * rz)], -1)


def conj(q):
    return q * q.new_tensor([-1.0, -1.0, -1.0, 1.0])


def d3_of(q):
    x, y, z, w = q.unbind(-1)
    return torch.stack([w * w + x * x - y * y - z * z, 2 * (x * y + w * z), 2 * (x * z - w * y)], -1)


def rotate(r, v):
    qv = r[..., :3]
    w = r[..., 3:4]
    a = w * v + torch.cross(qv.expand_as(v), v, dim=-1)
    c = (v * qv).sum(-1, keepdim=True)
    return w * a + torch.cross(qv.expand_as(a), a, dim=-1) + c * qv


class TorchVBD:
    """Holds the static set-up (float64 tensors) of one groom; `step` maps state tensors to state tensors."""

    def __init__(self, groom, material, *, num_itr, max_h, gravity, damping=1e-6, velocity_decay=0.05,
                 accel=1.0, sdf=None, body_rot=(0.0, 0.0, 0.0, 1.0), body_trans=(0.0, 0.0, 0.0),
                 wind=(0.0, 1.0, 0.7, 0.4, 3.0), ext_mult=1.0, time=0.0):
        t = lambda a: torch.as_tensor(np.asarray(a, np.float64))  # noqa: E731
        self.nv = groom.num_vertices
        sb = groom.strand_begin
        local = np.arange(self.nv) - np.repeat(sb[:-1], np.diff(sb))
        self.local = torch.as_tensor(local)
        self.im = t(material["inv_mass"])
        self.lr = t(material["l_rest"])
        self.ks = t(material["k_stretch"])
        fl = np.asarray(material["flags"], np.int64)
        self.hn = torch.as_tensor((fl & HAS_NEXT) != 0)
        self.hp = torch.as_tensor((fl & HAS_PREV) != 0)
        self.hno = torch.as_tensor((fl & HAS_NEXT_ORIENTATION) != 0)
        self.upd = torch.as_tensor(((fl & HAS_NEXT) != 0) & ((fl & FIX_ORIENTATION) == 0))
        self.root = torch.as_tensor(local == 0)
        self.num_itr, self.max_h = num_itr, max_h
        f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731  (the oracle takes C floats)
        self.g = t(f32(gravity))
        self.wind = [float(w) for w in f32(wind)]
        self.ext_mult = float(f32(ext_mult))
        self.time = float(np.float32(time))
        self.damping, self.decay, self.accel = float(f32(damping)), float(f32(velocity_decay)), float(f32(accel))
        self.sdf = sdf
        if sdf is not None:
            self.grid = torch.cat([t(sdf.grad).reshape(-1, 3), t(sdf.phi).reshape(-1, 1)], 1)
            self.dims = sdf.dims
            gmin = np.asarray(sdf.grid_min, np.float32).astype(np.float64)
            gmax = np.asarray(sdf.grid_max, np.float32).astype(np.float64)
            ds = (gmax - gmin) / np.asarray(sdf.dims, np.float64)  # as the FP64 oracle computes it
            self.gmin, self.ds = t(gmin), t(ds)
            self.inv = 1.0 / self.ds
            self.thresh = float(f32(sdf.threshold))
        self.rot = t(f32(body_rot))
        self.tr = t(f32(body_trans))

    @staticmethod
    def _shift_next(a):  # a[i+1] at i
        return torch.cat([a[1:], a[-1:]], 0)

    @staticmethod
    def _shift_prev(a):  # a[i-1] at i
        return torch.cat([a[:1], a[:-1]], 0)

    def _wind(self, x):
        """initItr's wind force along x: peak * max(0, pow(cY cZ, sharp) sign(cY cZ))."""
        peak, fy, fz, ft, sharp = self.wind
        ty = 2 * np.pi * (fy * x[:, 1] + ft * self.time)
        tz = 2 * np.pi * (fz * x[:, 2].abs() + ft * self.time)
        cy = torch.where(x[:, 1] > 0, torch.cos(ty), torch.zeros_like(ty))
        p = cy * torch.cos(tz)
        with torch.no_grad():
            on = torch.sign(p) * torch.pow(p, sharp) > 0  # NaN (negative base, fractional power) is off
        ps = torch.where(on, p, torch.ones_like(p))
        return torch.where(on, peak * torch.sign(ps) * torch.pow(ps, sharp), torch.zeros_like(p))

    def _predict(self, x, v, vl, h, last_h):
        free = (self.im != 0)[:, None]
        ext = self.g * self.ext_mult
        if self.wind[0] != 0.0:
            w = self._wind(x) * self.ext_mult
            ext = ext + torch.stack([w, torch.zeros_like(w), torch.zeros_like(w)], -1)
        dx = h * v
        y = torch.where(free, dx + h * h * ext, v)
        ext2 = (ext * ext).sum(-1)
        acc = (v - vl) / last_h
        s = torch.clamp((acc * ext).sum(-1) / ext2, 0.0, 1.0)
        dx = torch.where(free, dx + (h * h * s)[:, None] * ext, dx)
        return dx, y

    def _positions(self, x, dx, y, q, h, colour):
        damp = self.damping / h
        e = torch.where(self.hn[:, None], self._shift_next(x) - x, torch.zeros_like(x))
        invl = 1.0 / self.lr
        kk = self.ks * invl
        ddN = torch.where(self.hn, kk * invl, torch.zeros_like(kk))
        kkN = torch.where(self.hn, kk, torch.zeros_like(kk))
        ddP = torch.where(self.hp, self._shift_prev(ddN), torch.zeros_like(kk))
        kkP = torch.where(self.hp, self._shift_prev(kkN), torch.zeros_like(kk))
        free = self.im != 0
        a = torch.where(free, 1.0 / (self.im * h * h).clamp_min(1e-300), torch.zeros_like(kk))
        D = d3_of(q)
        dxN = self._shift_next(dx)
        dxP = self._shift_prev(dx)
        cN = (e + (dxN - dx)) * invl[:, None] - D
        eP = self._shift_prev(e)
        cP = (eP + (dx - dxP)) * self._shift_prev(invl)[:, None] - self._shift_prev(D)
        f = a[:, None] * (y - dx)
        f = f + kkN[:, None] * cN - (damp * ddN)[:, None] * dx
        f = f - kkP[:, None] * cP - (damp * ddP)[:, None] * dx
        s = (ddN + ddP) * (1 + damp)
        H = a[:, None, None] * torch.ones(3, 3, dtype=x.dtype) + s[:, None, None] * torch.eye(3, dtype=x.dtype)
        sel = free & ((self.local & 1) == colour)
        Hs = torch.where(sel[:, None, None], H, torch.eye(3, dtype=x.dtype).expand_as(H))
        delta = torch.linalg.solve(Hs, f[..., None])[..., 0]
        return torch.where(sel[:, None], dx + self.accel * delta, dx)

    def _orientations(self, x, dx, q, qr, colour):
        e = self._shift_next(x) - x
        V = -2.0 * self.ks[:, None] * (e + (self._shift_next(dx) - dx)) / self.lr[:, None]
        qP, qN = self._shift_prev(q), self._shift_next(q)
        qrP = self._shift_prev(qr)
        phi1 = torch.where((qmul(conj(qP), q) * qrP).sum(-1) > 0, 1.0, -1.0).to(q.dtype)
        phi2 = torch.where((qmul(conj(q), qN) * qr).sum(-1) > 0, 1.0, -1.0).to(q.dtype)
        b = torch.where(self.hp[:, None], phi1[:, None] * qmul(qP, qrP), torch.zeros_like(q))
        b = b + torch.where(self.hno[:, None], phi2[:, None] * qmul(qN, conj(qr)), torch.zeros_like(q))
        lam = torch.linalg.norm(V, dim=-1) + torch.linalg.norm(b, dim=-1)
        Vq = torch.cat([V, torch.zeros_like(V[:, :1])], -1)
        ex = q.new_tensor([1.0, 0.0, 0.0, 0.0]).expand_as(q)
        r = qmul(qmul(Vq, b), ex) + lam[:, None] * b
        sel = self.upd & ((self.local & 1) == colour)
        rs = torch.where(sel[:, None], r, q)
        return torch.where(sel[:, None], rs / torch.linalg.norm(rs, dim=-1, keepdim=True), q)

    def _sdf(self, x, v):
        nx, ny, nz = self.dims
        invq = conj(self.rot)
        lp = rotate(invq, x - self.tr) - self.gmin
        idx = torch.trunc((lp * self.inv).detach() + 0.5).long()
        inside = (idx[:, 0] >= 0) & (idx[:, 0] < nx) & (idx[:, 1] >= 0) & (idx[:, 1] < ny) & (idx[:, 2] >= 0) & (
            idx[:, 2] < nz)
        inside = inside & ~self.root
        ud = self.inv * (lp - (idx.to(x.dtype) - 0.5) * self.ds)
        res = 0
        for dz in (0, 1):
            for dy in (0, 1):
                for dxo in (0, 1):
                    c = idx + torch.tensor([dxo, dy, dz])
                    ok = (c[:, 0] < nx) & (c[:, 1] < ny) & (c[:, 2] < nz) & (c >= 0).all(-1)
                    cc = torch.stack([c[:, 0].clamp(0, nx - 1), c[:, 1].clamp(0, ny - 1), c[:, 2].clamp(0, nz - 1)], -1)
                    li = cc[:, 0] + nx * (cc[:, 1] + ny * cc[:, 2])
                    val = self.grid[li.clamp(0, self.grid.shape[0] - 1)]
                    val = torch.cat([torch.where(ok[:, None], val[:, :3], torch.zeros_like(val[:, :3])), val[:, 3:]], 1)
                    wx = ud[:, 0] if dxo else 1 - ud[:, 0]
                    wy = ud[:, 1] if dy else 1 - ud[:, 1]
                    wz = ud[:, 2] if dz else 1 - ud[:, 2]
                    res = res + (wx * wy * wz)[:, None] * val
        g = res[:, :3]
        n = g / torch.linalg.norm(g, dim=-1, keepdim=True).clamp_min(1e-300)
        phi = res[:, 3] - self.thresh
        hit = inside & (phi < 0)
        x2 = torch.where(hit[:, None], x - phi[:, None] * n, x)
        vn = torch.linalg.norm(v, dim=-1, keepdim=True)
        vhat = v / vn.clamp_min(1e-300)
        v2 = v - (vhat * n).sum(-1, keepdim=True) * n
        v2 = torch.where((hit & (vn[:, 0] >= 1e-6))[:, None], v2, v)
        return x2, v2

    def step(self, state, qr, dt):
        """state = (x, v, vl, q, h_prev) -> new state; qr is the (differentiable) rest Darboux array."""
        x, v, vl, q, h_prev = state
        steps = max(1, int(np.ceil(np.float32(dt) / np.float32(self.max_h))))
        h = float(np.float32(dt)) / steps  # as the FP64 oracle computes it
        last_h = h_prev
        for _ in range(steps):
            dx, y = self._predict(x, v, vl, h, last_h)
            vl = v
            for _it in range(self.num_itr):
                for c in (0, 1):
                    dx = self._positions(x, dx, y, q, h, c)
                for c in (0, 1):
                    q = self._orientations(x, dx, q, qr, c)
            free = (self.im != 0)[:, None]
            v = torch.where(free, dx * (1.0 / h) * (1 - self.decay * h), v)
            x = x + dx
        if self.sdf is not None:
            x, v = self._sdf(x, v)
        self.time = float(np.float32(self.time) + np.float32(dt))  # the solver's float clock
        return (x, v, vl, q, h)
