"""TEST INFRASTRUCTURE ONLY: a CPU restatement in float32 (numpy) of the
rendering passes of pbf_b200/csrc/pbf_render.cu, which restate the reference's
shaders (shaders/depth.vert, depth.frag, smooth.frag, thickness.frag,
normal.frag, background.frag, shadingParticle.frag; driven at
src/renderapp.cpp:400-466). Every float32 operation is taken in the order the
kernels take it, so the depth, smoothing, thickness, normal and room images
agree bit for bit; the shading pass calls exp and pow, whose last bits differ
between libraries, and is compared with a tolerance.

Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

F = np.float32
THICK_SCALE = F(16777216.0)
MAX_SPRITE = F(255.0)


def _row4(M, r, x, y, z):
    return ((M[r] * x + M[4 + r] * y) + M[8 + r] * z) + M[12 + r]


def _dot3(ax, ay, az, bx, by, bz):
    return (ax * bx + ay * by) + az * bz


def splat(cam, pos: np.ndarray, w: int, h: int):
    """(depth image with 0 where empty, thickness image) of particles pos [n, 3]."""
    V = np.array(cam.view[:], F)
    P = np.array(cam.proj[:], F)
    r = F(cam.radius)
    pc = F(cam.point_coeff)
    key = np.full(w * h, np.iinfo(np.uint64).max, np.uint64)
    acc = np.zeros(w * h, np.int64)
    pos = np.asarray(pos, F)
    for px, py, pz in pos:
        vx, vy, vz = _row4(V, 0, px, py, pz), _row4(V, 1, px, py, pz), _row4(V, 2, px, py, pz)
        if not vz < 0:
            continue
        cx, cy, cz, cw = (_row4(P, k, vx, vy, vz) for k in range(4))
        if not cw > 0:
            continue
        ndz = cz / cw
        if not (ndz >= -1 and ndz <= 1):
            continue
        wx = (cx / cw + F(1)) * F(0.5) * F(w)
        wy = (cy / cw + F(1)) * F(0.5) * F(h)
        size = -pc * r / vz
        size = min(max(size, F(1)), MAX_SPRITE)
        half = F(0.5) * size
        if not (wx + half >= 0 and wx - half <= F(w) and wy + half >= 0 and wy - half <= F(h)):
            continue
        x0 = max(int(np.ceil(wx - half - F(0.5))), 0)
        x1 = min(int(np.ceil(wx + half - F(0.5))) - 1, w - 1)
        y0 = max(int(np.ceil(wy - half - F(0.5))), 0)
        y1 = min(int(np.ceil(wy + half - F(0.5))) - 1, h - 1)
        for yy in range(y0, y1 + 1):
            for xx in range(x0, x1 + 1):
                s = (F(xx) + F(0.5) - wx) / size + F(0.5)
                t = F(0.5) - (F(yy) + F(0.5) - wy) / size
                nx = F(2) * s + F(-1)
                ny = F(-2) * t + F(1)
                d2 = nx * nx + ny * ny
                if d2 > 1:
                    continue
                nz = np.sqrt(F(1) - d2)
                pix = yy * w + xx
                th = F(2) * nz * r
                acc[pix] += int(np.rint(th * THICK_SCALE))
                sx, sy, sz = vx + r * nx, vy + r * ny, vz + r * nz
                qz, qw = _row4(P, 2, sx, sy, sz), _row4(P, 3, sx, sy, sz)
                fd = F(0.5) * (qz / qw) + F(0.5)
                fd = min(max(fd, F(0)), F(1))
                k = (np.uint64(np.array(fd, F).view(np.uint32)) << np.uint64(32)) | np.uint64(np.array(-sz, F).view(np.uint32))
                if k < key[pix]:
                    key[pix] = k
    empty = key == np.iinfo(np.uint64).max
    z = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(F)
    z = np.where(empty, F(0), z).astype(F)
    thick = acc.astype(F) * (F(1) / THICK_SCALE)
    return z.reshape(h, w), thick.reshape(h, w)


def _sh(a, dx, dy):
    """texel (x + dx, y + dy) with GL_REPEAT wrapping; a is [h, w]"""
    return np.roll(np.roll(a, -dy, axis=0), -dx, axis=1)


def smooth(z: np.ndarray, Fx, Fy, iterations: int) -> np.ndarray:
    h, w = z.shape
    Cx = F(2) / (F(w) * F(Fx))
    Cy = F(2) / (F(h) * F(Fy))
    with np.errstate(all="ignore"):
        for _ in range(iterations):
            zpx, zmx, zpy, zmy = _sh(z, 1, 0), _sh(z, -1, 0), _sh(z, 0, 1), _sh(z, 0, -1)
            dzdx = np.where((zpx == 0) | (zmx == 0), F(0), (zpx - zmx) * F(0.5))
            dz2dx2 = (zpx + zmx) - F(2) * z
            dzdy = np.where((zpy == 0) | (zmy == 0), F(0), (zpy - zmy) * F(0.5))
            dz2dy2 = (zpy + zmy) - F(2) * z
            zpp, zpm, zmp, zmm = _sh(z, 1, 1), _sh(z, 1, -1), _sh(z, -1, 1), _sh(z, -1, -1)
            dz2dxdy = (((zpp + zmm) - zmp) - zpm) * F(0.25)
            nx, ny, nz = -Cy * dzdx, Cx * dzdy, (Cx * Cy) * z
            D = _dot3(nx, ny, nz, nx, ny, nz)
            Cx2, Cy2 = Cx * Cx, Cy * Cy
            dDdx = F(2) * (((Cy2 * dzdx) * dz2dx2 + (Cx2 * dzdy) * dz2dxdy) + ((Cx2 * Cy2) * z) * dzdx)
            dDdy = F(2) * (((Cy2 * dzdx) * dz2dxdy + (Cx2 * dzdy) * dz2dy2) + ((Cx2 * Cy2) * z) * dzdy)
            Ex = (F(0.5) * dzdx) * dDdx - dz2dx2 * D
            Ey = (F(0.5) * dzdy) * dDdy - dz2dy2 * D
            H = (F(0.5) * (Cy * Ex + Cx * Ey)) / (D * np.sqrt(D))
            out = z - H * F(0.01)
            out = np.where(out < 0, z, out)
            z = np.where(z > 0, out, F(0)).astype(F)
    return z


def normals(z: np.ndarray, Fx, Fy) -> np.ndarray:
    h, w = z.shape
    Cx = F(2) / (F(w) * F(Fx))
    Cy = F(2) / (F(h) * F(Fy))
    zpx, zmx, zpy, zmy = _sh(z, 1, 0), _sh(z, -1, 0), _sh(z, 0, 1), _sh(z, 0, -1)
    with np.errstate(all="ignore"):
        dzdx = np.where((zpx == 0) | (zmx == 0), F(0), (zpx - zmx) * F(0.5))
        dzdy = np.where((zpy == 0) | (zmy == 0), F(0), (zpy - zmy) * F(0.5))
        nx, ny, nz = -Cy * dzdx, Cx * dzdy, (Cx * Cy) * z
        ln = np.sqrt(_dot3(nx, ny, nz, nx, ny, nz))
        out = np.stack([nx / ln, ny / ln, nz / ln, np.zeros_like(z)], axis=-1)
    return np.where((z > 0)[..., None], out, F(0)).astype(F)


def _quant8(v):
    return (np.rint(np.clip(v, F(0), F(1)) * F(255)) / F(255)).astype(F)


def room(cam, w: int, h: int) -> np.ndarray:
    V = np.array(cam.view[:], F)
    P = np.array(cam.proj[:], F)
    eye = np.array(cam.cam_pos[:], F)
    R = np.array(cam.room[:], F)
    xs = np.arange(w, dtype=F)[None, :].repeat(h, 0)
    ys = np.arange(h, dtype=F)[:, None].repeat(w, 1)
    ux = (F(2) * (xs + F(0.5)) / F(w) - F(1)) / P[0]
    uy = (F(2) * (ys + F(0.5)) / F(h) - F(1)) / P[5]
    d = [(V[4 * a] * ux + V[4 * a + 1] * uy) - V[4 * a + 2] for a in range(3)]
    best = np.full((h, w), F(3.4e38), F)
    nrm = np.zeros((3, h, w), F)
    with np.errstate(all="ignore"):
        for a, v, ns in ((0, R[0], 1.0), (0, R[3], -1.0), (1, R[1], 1.0), (2, R[2], 1.0)):
            t = (v - eye[a]) / d[a]
            b, e = (a + 1) % 3, (a + 2) % 3
            pb = eye[b] + t * d[b]
            pe = eye[e] + t * d[e]
            ok = (d[a] != 0) & (t > 0) & (t < best) & ~((pb < R[b]) | (pb > R[3 + b]) | (pe < R[e]) | (pe > R[3 + e]))
            best = np.where(ok, t, best)
            for k in range(3):
                nrm[k] = np.where(ok, F(ns) if k == a else F(0), nrm[k])
        hit = best < F(3.4e38)
        p = [eye[k] + best * d[k] for k in range(3)]
        L = np.array(cam.room_light_pos[:], F)
        Ld = np.array(cam.room_light_diffuse[:], F)
        lx, ly, lz = L[0] - p[0], L[1] - p[1], L[2] - p[2]
        ll = np.sqrt(_dot3(lx, ly, lz, lx, ly, lz))
        lx, ly, lz = lx / ll, ly / ll, lz / ll
        diff = np.maximum(_dot3(lx, ly, lz, nrm[0], nrm[1], nrm[2]), F(0))
    out = np.ones((h, w, 4), F)
    for k in range(3):
        out[..., k] = _quant8(np.where(hit, F(0.2) + (diff * Ld[k]) * F(0.95), F(0.75)))
    return out


def shade(cam, z, thick, nrm, bg) -> np.ndarray:
    h, w = z.shape
    V = np.array(cam.view[:], F)
    xs = np.arange(w, dtype=F)[None, :].repeat(h, 0)
    ys = np.arange(h, dtype=F)[:, None].repeat(w, 1)
    u = (xs + F(0.5)) / F(w)
    v = (ys + F(0.5)) / F(h)
    th = F(cam.tan_half_fov)
    with np.errstate(all="ignore"):
        sx, sy, sz = (F(2) * u - F(1)) * th * z, (F(2) * v - F(1)) * th * z, -z
        vx, vy, vz = -sx, -sy, -sz
        vl = np.sqrt(_dot3(vx, vy, vz, vx, vy, vz))
        vx, vy, vz = vx / vl, vy / vl, vz / vl
        L = np.array(cam.light_pos[:], F)
        lp = [_row4(V, k, L[0], L[1], L[2]) for k in range(3)]
        lx, ly, lz = lp[0] - sx, lp[1] - sy, lp[2] - sz
        ll = np.sqrt(_dot3(lx, ly, lz, lx, ly, lz))
        lx, ly, lz = lx / ll, ly / ll, lz / ll
        nx, ny, nz = nrm[..., 0], nrm[..., 1], nrm[..., 2]
        thickness = F(0.08) * thick
        beta = F(0.01) * thickness
        bx = np.floor((u + beta * nx) * F(w)).astype(np.int64) % w
        by = np.floor((v + beta * ny) * F(h)).astype(np.int64) % h
        S = bg[by, bx]
        e = np.exp(-thickness).astype(F)
        cf = [F(0.1), F(0.4), F(0.8)]
        cosv = np.clip(_dot3(nx, ny, nz, vx, vy, vz), F(0), F(1))
        f = (F(1) - F(cam.roi)) / (F(1) + F(cam.roi))
        FF = f * f
        Fr = FF * (F(1) - FF) * np.power(F(1) - cosv, F(5))
        diff = np.maximum(_dot3(lx, ly, lz, nx, ny, nz), F(0))
        dn = _dot3(nx, ny, nz, -lx, -ly, -lz)
        rx, ry, rz = -lx - F(2) * dn * nx, -ly - F(2) * dn * ny, -lz - F(2) * dn * nz
        spec = np.power(np.maximum(_dot3(vx, vy, vz, rx, ry, rz), F(0)), F(32))
        Ld = np.array(cam.light_diffuse[:], F)
        out = np.ones((h, w, 4), F)
        for k in range(3):
            a = cf[k] * (F(1) - e) + S[..., k] * e
            out[..., k] = (a * (F(1) - Fr) + ((diff * Ld[k]) * cf[k]) * Fr) + spec
    return np.where((z > 0)[..., None], out, bg).astype(F)


def render(cam, pos, w, h):
    """All images: dict depth_raw, depth, thickness, normal, room, color."""
    z0, thick = splat(cam, pos, w, h)
    Fy, Fx = cam.proj[0], cam.proj[5]
    z = smooth(z0, Fx, Fy, cam.smooth_iterations)
    n = normals(z, Fx, Fy)
    bg = room(cam, w, h)
    return {"depth_raw": z0, "depth": z, "thickness": thick, "normal": n, "room": bg,
            "color": shade(cam, z, thick, n, bg)}
