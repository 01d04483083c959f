"""Known answers for the rendering restatement (oracle/render_oracle.py), which the
CUDA passes (pbf_b200/csrc/pbf_render.cu) match bit for bit on real scenes
(tests/test_gpu_render.py). The reference's OpenGL passes cannot run on these
machines, so each pass is pinned to what its shader computes, worked out in
float64 from the shader's text on inputs whose answer is known in closed form:

* depth.vert / depth.frag / thickness.frag: a point sprite of
  pointCoeff * radius / |z_view| pixels covers the pixels whose centres fall in
  its disc; each writes the sphere's front |z_view| - r sqrt(1 - rho^2) and its
  chord 2 r sqrt(1 - rho^2). Depth goes through the depth test
  (src/renderapp.cpp:406), thickness is blended additively with no depth test
  (:428-433).
* smooth.frag: one explicit step z - 0.01 H of screen-space curvature flow, H
  in closed form for ramps and a paraboloid; a flat interior stays as it is.
  Textures are read with GL_NEAREST and the default GL_REPEAT (the app sets no
  wrap mode, :302-331).
* normal.frag: normalize(-Cy dz/dx, Cx dz/dy, Cx Cy z), with z the positive
  distance the depth pass writes.
* background.frag: ambient 0.2 plus the room light's diffuse term times the
  wall colour 0.95, stored in an 8-bit RGBA texture (:329); 0.75 where no wall
  is drawn (:449).
* shadingParticle.frag: Beer-Lambert mix of the fluid colour and the refracted
  background, Schlick's Fresnel term, Lambert diffuse and a Phong highlight.

These run on the CPU: they pin the oracle, and through it the kernels.
"""
import math

import numpy as np

from oracle import render_oracle as RO
from pbf_b200 import render

F32 = np.float32


def _sprite_camera(w, h, dist, radius, fovy_deg=30.0, light=(0.0, 50.0, -20.0)):
    return render.make_camera((0.0, 0.0, dist), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), math.radians(fovy_deg), w, h,
                              radius, smooth_iterations=0, light=light)


def _window_pos(cam, p, w, h):
    """(window x, window y, distance in front of the camera) of world point p, in float64."""
    V = np.array(cam.view[:], np.float64).reshape(4, 4).T
    P = np.array(cam.proj[:], np.float64).reshape(4, 4).T
    vp = V @ np.array([p[0], p[1], p[2], 1.0])
    c = P @ vp
    return (c[0] / c[3] + 1.0) * 0.5 * w, (c[1] / c[3] + 1.0) * 0.5 * h, -vp[2]


def _sphere_profile(cam, w, h, p=(0.0, 0.0, 0.0)):
    """(covered, rho^2, depth, chord) of the sprite of the particle at world p."""
    cx, cy, dist = _window_pos(cam, p, w, h)
    size = float(cam.point_coeff) * float(cam.radius) / dist
    xs = np.arange(w)[None, :] + 0.5
    ys = np.arange(h)[:, None] + 0.5
    nx = 2.0 * (xs - cx) / size
    ny = 2.0 * (ys - cy) / size
    rho2 = nx * nx + ny * ny
    covered = rho2 <= 1.0
    nz = np.sqrt(np.clip(1.0 - rho2, 0.0, None))
    r = float(cam.radius)
    return covered, rho2, dist - r * nz, 2.0 * r * nz


def test_sprite_depth_and_thickness_are_the_sphere_front_and_chord():
    w = h = 129
    dist, r = 5.0, 0.5
    cam = _sprite_camera(w, h, dist, r)
    z, th = RO.splat(cam, np.zeros((1, 3), F32), w, h)
    covered, rho2, depth, chord = _sphere_profile(cam, w, h)
    clear = np.abs(rho2 - 1.0) > 1e-4  # pixels not on the rim, where rounding decides
    assert np.array_equal((z > 0)[clear], covered[clear])
    assert np.array_equal((th > 0)[clear], covered[clear])
    inside = rho2 < 0.99  # where sqrt(1 - rho^2) is not sensitive to the last bit of rho^2
    assert inside.sum() > 1500
    assert np.abs(z[inside] - depth[inside]).max() <= 1e-6 * dist
    assert np.abs(th[inside] - chord[inside]).max() <= 1e-6
    assert np.all(z[~covered & clear] == 0) and np.all(th[~covered & clear] == 0)


def test_thickness_integrates_to_the_sphere_volume():
    """Each pixel of the sprite is 2r / size wide at the sphere, so the chords
    sum to the volume 4/3 pi r^3 (the disc's rim is resolved to a pixel)."""
    w = h = 161
    dist, r = 3.0, 0.5
    cam = _sprite_camera(w, h, dist, r)
    _, th = RO.splat(cam, np.zeros((1, 3), F32), w, h)
    size = float(cam.point_coeff) * r / dist
    assert size > 70
    vol = float(th.astype(np.float64).sum()) * (2.0 * r / size) ** 2
    assert abs(vol / (4.0 / 3.0 * math.pi * r ** 3) - 1.0) < 5e-3


def test_coincident_and_overlapping_sprites():
    """Thickness adds over sprites whatever their depth; depth keeps the nearest
    front at every pixel (two overlapping spheres of radius 0.5, the second 0.3
    farther and off the axis: its front comes through near the first's rim)."""
    w = h = 129
    dist, r = 5.0, 0.5
    cam = _sprite_camera(w, h, dist, r)
    z1, th1 = RO.splat(cam, np.zeros((1, 3), F32), w, h)
    z5, th5 = RO.splat(cam, np.zeros((5, 3), F32), w, h)
    assert np.array_equal(z5, z1)
    assert np.allclose(th5, 5.0 * th1.astype(np.float64), rtol=2.0 ** -21, atol=0.0)

    second = (0.6, 0.1, -0.3)
    pos = np.array([[0.0, 0.0, 0.0], second], F32)
    z, th = RO.splat(cam, pos, w, h)
    c1, q1, d1, t1 = _sphere_profile(cam, w, h)
    c2, q2, d2, t2 = _sphere_profile(cam, w, h, second)
    inside = ((q1 < 0.99) | (q1 > 1.01)) & ((q2 < 0.99) | (q2 > 1.01))
    want_z = np.where(c1 & c2, np.minimum(d1, d2), np.where(c1, d1, np.where(c2, d2, 0.0)))
    want_t = np.where(c1, t1, 0.0) + np.where(c2, t2, 0.0)
    # the off-axis sprite's window position carries float32 rounding of the
    # projection (about 1e-5 pixel), which moves rho^2 by about 1e-6
    assert np.abs(z[inside] - want_z[inside]).max() <= 2e-6 * dist
    assert np.abs(th[inside] - want_t[inside]).max() <= 1e-5
    both = c1 & c2 & inside
    assert (both & (d2 < d1)).sum() > 20 and (both & (d1 < d2)).sum() > 20  # each front wins somewhere


# ---------------------------------------------------------------------------
# smooth.frag and normal.frag
# ---------------------------------------------------------------------------
def _smooth_step_f64(z, Fx, Fy):
    """One pass of smooth.frag in float64, texel by texel (GL_REPEAT, nearest)."""
    h, w = z.shape
    Cx = 2.0 / (w * Fx)
    Cy = 2.0 / (h * Fy)
    zz = z.astype(np.float64)
    out = np.zeros_like(zz)

    def at(x, y):
        return zz[y % h, x % w]

    for y in range(h):
        for x in range(w):
            c = zz[y, x]
            if not c > 0:
                continue
            zpx, zmx, zpy, zmy = at(x + 1, y), at(x - 1, y), at(x, y + 1), at(x, y - 1)
            dzdx = 0.0 if (zpx == 0 or zmx == 0) else (zpx - zmx) * 0.5
            dzdy = 0.0 if (zpy == 0 or zmy == 0) else (zpy - zmy) * 0.5
            dz2dx2 = zpx + zmx - 2.0 * c
            dz2dy2 = zpy + zmy - 2.0 * c
            dz2dxdy = (at(x + 1, y + 1) + at(x - 1, y - 1) - at(x - 1, y + 1) - at(x + 1, y - 1)) * 0.25
            n = np.array([-Cy * dzdx, Cx * dzdy, Cx * Cy * c])
            D = float(n @ n)
            dDdx = 2.0 * (Cy * Cy * dzdx * dz2dx2 + Cx * Cx * dzdy * dz2dxdy + Cx * Cx * Cy * Cy * c * dzdx)
            dDdy = 2.0 * (Cy * Cy * dzdx * dz2dxdy + Cx * Cx * dzdy * dz2dy2 + Cx * Cx * Cy * Cy * c * dzdy)
            Ex = 0.5 * dzdx * dDdx - dz2dx2 * D
            Ey = 0.5 * dzdy * dDdy - dz2dy2 * D
            H = 0.5 * (Cy * Ex + Cx * Ey) / (D * math.sqrt(D))
            s = c - H * 0.01
            out[y, x] = c if s < 0 else s
    return out


def _curvature_at_spike(zc, zn, w, h):
    """H at a texel of depth zc whose eight neighbours are all zn: dz/dx = dz/dy
    = 0, d2z/dx2 = d2z/dy2 = 2 (zn - zc), so H = (zc - zn)(Cx + Cy) / (Cx Cy zc)."""
    Cx, Cy = 2.0 / (w * FX), 2.0 / (h * FY)
    return (zc - zn) * (Cx + Cy) / (Cx * Cy * zc)


def _normals_f64(z, Fx, Fy):
    h, w = z.shape
    Cx = 2.0 / (w * Fx)
    Cy = 2.0 / (h * Fy)
    zz = z.astype(np.float64)
    out = np.zeros((h, w, 3))
    for y in range(h):
        for x in range(w):
            c = zz[y, x]
            if not c > 0:
                continue
            zpx, zmx = zz[y, (x + 1) % w], zz[y, (x - 1) % w]
            zpy, zmy = zz[(y + 1) % h, x], zz[(y - 1) % h, x]
            dzdx = 0.0 if (zpx == 0 or zmx == 0) else (zpx - zmx) * 0.5
            dzdy = 0.0 if (zpy == 0 or zmy == 0) else (zpy - zmy) * 0.5
            n = np.array([-Cy * dzdx, Cx * dzdy, Cx * Cy * c])
            out[y, x] = n / np.linalg.norm(n)
    return out


def _close_step(got, want, z0, rel=1e-2):
    """The step z' - z agrees to `rel` of itself plus float32 rounding of z."""
    dg = got.astype(np.float64) - z0.astype(np.float64)
    dw = want - z0.astype(np.float64)
    return np.abs(dg - dw) <= rel * np.abs(dw) + 4.0 * np.spacing(np.abs(z0).astype(F32)).astype(np.float64)


FX, FY = 0.5, 0.625  # small frusta: Cx, Cy of a few tenths, so steps are far above rounding


def test_smoothing_leaves_a_flat_interior_unchanged():
    w = h = 48
    z = np.zeros((h, w), F32)
    z[8:40, 6:42] = F32(0.75)
    out = RO.smooth(z, FX, FY, 5)
    assert np.array_equal(out[14:34, 12:36], z[14:34, 12:36])  # 6 texels from every edge
    assert np.all(out[z == 0] == 0)
    assert not np.array_equal(out[8], z[8])  # the rim moves


def test_smoothing_step_on_ramps_and_a_paraboloid():
    w, h = 24, 20
    Cx, Cy = 2.0 / (w * FX), 2.0 / (h * FY)
    xs = np.arange(w, dtype=np.float64)[None, :].repeat(h, 0)
    ys = np.arange(h, dtype=np.float64)[:, None].repeat(w, 1)
    z0 = 0.05
    # x ramp, b = sqrt(2) Cx z0 (where H is largest): H = Cx^2 Cy^3 z b^2 / (2 D^1.5), D = Cy^2 b^2 + Cx^2 Cy^2 z^2
    b = math.sqrt(2.0) * Cx * z0 / 8.0
    z = (z0 + b * (xs - w / 2)).astype(F32)
    got = RO.smooth(z, FX, FY, 1)
    zf = z.astype(np.float64)
    D = Cy * Cy * b * b + Cx * Cx * Cy * Cy * zf * zf
    want = zf - 0.01 * (0.5 * Cx * Cx * Cy ** 3 * zf * b * b / D ** 1.5)
    inner = (xs >= 1) & (xs <= w - 2)  # the ramp wraps at the image's left and right edges
    assert _close_step(got, want, z)[inner].all()
    assert (np.abs(want - zf)[inner] > 1e-6).all()
    # y ramp: H = Cx^3 Cy^2 z b^2 / (2 D^1.5), D = Cx^2 b^2 + Cx^2 Cy^2 z^2
    b = math.sqrt(2.0) * Cy * z0 / 8.0
    z = (z0 + b * (ys - h / 2)).astype(F32)
    got = RO.smooth(z, FX, FY, 1)
    zf = z.astype(np.float64)
    D = Cx * Cx * b * b + Cx * Cx * Cy * Cy * zf * zf
    want = zf - 0.01 * (0.5 * Cx ** 3 * Cy * Cy * zf * b * b / D ** 1.5)
    inner = (ys >= 1) & (ys <= h - 2)
    assert _close_step(got, want, z)[inner].all()
    # paraboloid z0 + c ((x - 12)^2 + (y - 10)^2) / 2, exact in float32 near its apex:
    # at the apex H = -c (Cx + Cy) / (2 Cx Cy z0), so the apex moves back by 0.005 c (Cx + Cy) / (Cx Cy z0)
    c = 2.0 ** -9
    z = (0.5 + 0.5 * c * ((xs - 12) ** 2 + (ys - 10) ** 2)).astype(F32)
    got = RO.smooth(z, FX, FY, 1)
    step = 0.005 * c * (Cx + Cy) / (Cx * Cy * 0.5)
    assert abs((float(got[10, 12]) - 0.5) - step) <= 1e-3 * step + 4.0 * float(np.spacing(F32(0.5)))


def test_smoothing_matches_the_shader_in_float64_with_holes_and_wrap():
    """A bumpy field touching all four image edges, with holes: the one-sided
    derivative rule beside empty texels, the repeat wrap at the edges, and the
    rule that keeps z where the step would make it negative."""
    rng = np.random.RandomState(3)
    w, h = 28, 22
    xs = np.arange(w)[None, :]
    ys = np.arange(h)[:, None]
    z = 0.3 + 0.02 * np.sin(2 * math.pi * xs / w) * np.cos(2 * math.pi * ys / h) + 0.004 * rng.rand(h, w)
    z[rng.rand(h, w) < 0.08] = 0.0
    z[4:7, 6:9] = 1e-3
    z[5, 7] = 0.05  # a spike away from the camera among near-zero texels: its step would go below zero
    z = z.astype(F32)
    got = RO.smooth(z, FX, FY, 1)
    want = _smooth_step_f64(z, FX, FY)
    assert np.all((got == 0) == (z == 0))
    ok = _close_step(got, want, z)
    assert ok.all(), np.argwhere(~ok)[:5]
    assert got[5, 7] == z[5, 7] and want[5, 7] == z[5, 7]
    assert 0.05 - 0.01 * _curvature_at_spike(0.05, 1e-3, w, h) < 0
    assert (np.abs(want - z)[z > 0] > 1e-5).mean() > 0.5


def test_normals_flat_ramp_and_orientation():
    w, h = 24, 20
    Cx, Cy = 2.0 / (w * FX), 2.0 / (h * FY)
    z = np.full((h, w), F32(0.4))
    n = RO.normals(z, FX, FY)
    assert np.all(n[..., :3] == np.float32([0.0, 0.0, 1.0])) and np.all(n[..., 3] == 0)
    # x ramp: (-Cy b, 0, Cx Cy z) / |.|
    xs = np.arange(w, dtype=np.float64)[None, :].repeat(h, 0)
    b = 0.01
    z = (0.4 + b * (xs - w / 2)).astype(F32)
    n = RO.normals(z, FX, FY)
    zf = z.astype(np.float64)
    L = np.sqrt(Cy * Cy * b * b + (Cx * Cy * zf) ** 2)
    inner = (xs >= 1) & (xs <= w - 2)
    assert np.abs(n[..., 0] - (-Cy * b / L))[inner].max() < 1e-5
    assert np.abs(n[..., 2] - (Cx * Cy * zf / L))[inner].max() < 1e-5
    assert np.all(n[..., 1][inner] == 0)
    # the shader's formula on a field with holes
    rng = np.random.RandomState(5)
    z = (0.3 + 0.05 * rng.rand(h, w)).astype(F32)
    z[rng.rand(h, w) < 0.1] = 0
    n = RO.normals(z, FX, FY)
    assert np.abs(n[..., :3] - _normals_f64(z, FX, FY)).max() < 1e-5
    # on a sprite: the y component points up on the upper half and, with z the
    # positive distance in the shader's -Cy dz/dx, the x component points to -x
    # on the right half (the reference's sign convention, kept)
    W = 97
    cam = _sprite_camera(W, W, 5.0, 0.5)
    zs, _ = RO.splat(cam, np.zeros((1, 3), F32), W, W)
    ns = RO.normals(zs, cam.proj[5], cam.proj[0])
    c = W // 2
    row, col = ns[c, c + 3:c + 10], ns[c + 3:c + 10, c]
    assert np.all(row[:, 0] < 0) and np.all(col[:, 1] > 0)
    assert np.all(ns[c, c - 10:c - 3, 0] > 0) and np.all(ns[c - 10:c - 3, c, 1] < 0)


# ---------------------------------------------------------------------------
# background.frag (the room) and shadingParticle.frag
# ---------------------------------------------------------------------------
def _q8(v):
    return np.rint(np.clip(v, 0.0, 1.0) * 255.0) / 255.0


def _room_centre(eye, target, up):
    w = h = 33
    cam = render.make_camera(eye, target, up, math.radians(40.0), w, h, 0.1)
    return RO.room(cam, w, h)[h // 2, w // 2]


def test_room_walls_floor_and_open_sides():
    light = np.array([0.0, 50.0, 0.0])  # the room light (src/renderapp.cpp:110)

    def lit(p, n):
        d = light - np.asarray(p, float)
        diff = max(float(d @ np.asarray(n, float)) / np.linalg.norm(d), 0.0)
        return _q8(0.2 + diff * 0.8 * 0.95)

    cases = [  # eye, target, up, the wall point the centre ray meets, its normal
        ((0.0, 25.0, 20.0), (0.0, 25.0, -30.0), (0, 1, 0), (0.0, 25.0, -30.0), (0, 0, 1)),   # back wall
        ((5.0, 30.0, 5.0), (5.0, 0.0, 5.0), (0, 0, -1), (5.0, 0.0, 5.0), (0, 1, 0)),         # floor
        ((0.0, 10.0, 0.0), (30.0, 10.0, 0.0), (0, 1, 0), (30.0, 10.0, 0.0), (-1, 0, 0)),     # right wall
        ((0.0, 40.0, 4.0), (-30.0, 40.0, 4.0), (0, 1, 0), (-30.0, 40.0, 4.0), (1, 0, 0)),    # left wall
    ]
    for eye, target, up, p, n in cases:
        got = _room_centre(eye, target, up)
        want = lit(p, n)
        assert np.all(got[:3] == np.float32(want)), (eye, got, want)
        assert got[3] == 1.0
    # the front and the top are open: the clear colour 0.75
    for eye, target, up in (((0.0, 25.0, 0.0), (0.0, 25.0, 30.0), (0, 1, 0)),
                            ((0.0, 25.0, 0.0), (0.0, 60.0, 0.0), (0, 0, -1))):
        got = _room_centre(eye, target, up)
        assert np.all(got[:3] == np.float32(_q8(0.75)))


def test_shading_closed_forms():
    w, h = 33, 21
    eye = (0.0, 0.0, 5.0)
    cam = _sprite_camera(w, h, 5.0, 0.1, light=eye)  # the light at the eye: it shines along the view axis
    cf = np.array([0.1, 0.4, 0.8])
    cx, cy = w // 2, h // 2
    z = np.zeros((h, w), F32)
    thick = np.zeros((h, w), F32)
    nrm = np.zeros((h, w, 4), F32)
    bg = np.ones((h, w, 4), F32)
    bg[..., 0] = (np.arange(w) / 64.0)[None, :]  # a colour per column, to find the refracted texel
    bg[..., 1] = 0.5
    bg[..., 2] = (np.arange(h) / 64.0)[:, None]
    # (a) the centre texel facing the eye, no fluid thickness: the background,
    #     no Fresnel term (cos = 1), full diffuse times F = 0, specular 1
    z[cy, cx] = 2.0
    nrm[cy, cx, 2] = 1.0
    # (b) a texel beside it, thick fluid: the fluid colour instead of the background
    z[cy, cx + 1] = 2.0
    nrm[cy, cx + 1, 2] = 1.0
    thick[cy, cx + 1] = 1e4
    # (c) the centre column one row up... seen edge-on: n = (1, 0, 0) on the view axis
    #     needs the centre texel, so use a second image for it below
    out = RO.shade(cam, z, thick, nrm, bg)
    assert np.abs(out[cy, cx, :3] - (bg[cy, cx, :3] + 1.0)).max() < 1e-6
    # (b) is one texel right of the axis: v and the light direction tilt by
    # atan(2 tanHalfFov / w); Fresnel and the highlight follow from them
    u = (cx + 1 + 0.5) / w
    sx = (2 * u - 1) * float(cam.tan_half_fov) * 2.0
    s = np.array([sx, 0.0, -2.0])
    v = -s / np.linalg.norm(s)
    ld = v  # the light is at the eye
    cosv = min(max(v[2], 0.0), 1.0)
    f = (1 - 1.3) / (1 + 1.3)
    Fr = f * f * (1 - f * f) * (1 - cosv) ** 5
    diff = max(ld[2], 0.0)
    r = -ld - 2.0 * float(np.array([0, 0, 1.0]) @ -ld) * np.array([0, 0, 1.0])
    spec = max(float(v @ r), 0.0) ** 32
    want = cf * (1 - Fr) + diff * 0.8 * cf * Fr + spec
    assert np.abs(out[cy, cx + 1, :3] - want).max() < 2e-6
    # empty texels show the room
    assert np.array_equal(out[0, 0], bg[0, 0]) and np.array_equal(out[cy + 1, cx], bg[cy + 1, cx])

    # (c) edge-on at the centre texel: cos = 0, so F = f^2 (1 - f^2); the light
    #     along the view axis gives no diffuse and no highlight; the background
    #     is read beta n.x = 3 texels to the right
    z = np.zeros((h, w), F32)
    nrm = np.zeros((h, w, 4), F32)
    thick = np.zeros((h, w), F32)
    z[cy, cx] = 2.0
    nrm[cy, cx, 0] = 1.0
    t = 3.0 / (w * 0.01 * 0.08)
    thick[cy, cx] = t
    out = RO.shade(cam, z, thick, nrm, bg)
    e = math.exp(-0.08 * t)
    S = bg[cy, cx + 3, :3].astype(np.float64)
    a = cf * (1 - e) + S * e
    Fr = f * f * (1 - f * f)
    assert np.abs(out[cy, cx, :3] - a * (1 - Fr)).max() < 2e-6
    # the same at the right edge: the refracted read wraps to column 1
    z = np.zeros((h, w), F32)
    z[cy, w - 2] = 2.0
    out = RO.shade(cam, z, np.roll(thick, w - 2 - cx, axis=1), np.roll(nrm, w - 2 - cx, axis=1), bg)
    got_col = out[cy, w - 2, :3]
    u = (w - 2 + 0.5) / w
    s = np.array([(2 * u - 1) * float(cam.tan_half_fov) * 2.0, 0.0, -2.0])
    v = -s / np.linalg.norm(s)
    cosv = min(max(v[0], 0.0), 1.0)  # dot(n, v) with n = (1, 0, 0)
    Fr = f * f * (1 - f * f) * (1 - cosv) ** 5
    diff = max(v[0], 0.0)  # dot(lightDir, n), lightDir = v
    r = -v - 2.0 * float(np.array([1.0, 0, 0]) @ -v) * np.array([1.0, 0, 0])
    spec = max(float(v @ r), 0.0) ** 32
    S = bg[cy, 1, :3].astype(np.float64)
    a = cf * (1 - e) + S * e
    want = a * (1 - Fr) + diff * 0.8 * cf * Fr + spec
    assert np.abs(got_col - want).max() < 2e-6
