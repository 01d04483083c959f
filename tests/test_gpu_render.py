"""Headless rendering: the CUDA passes (pbf_b200/csrc/pbf_render.cu) against the
float32 restatement of the reference's shaders (oracle/render_oracle.py).
Depth, smoothing, thickness, normals and the room are compared bit for bit;
the shading (exp, pow) within 2e-5."""
import math

import numpy as np
import pytest

from oracle import render_oracle as RO
from pbf_b200 import render, scenes


def _blob(n=400, seed=0):
    rng = np.random.RandomState(seed)
    c = np.array([0.5, 0.3, 0.4])
    return (c + rng.normal(scale=0.12, size=(n, 3))).astype(np.float32)


def _cam(w, h, iters=6, radius=0.03):
    return render.box_camera((0.0, 0.0, 0.0, 1.0, 0.8, 0.8), w, h, radius, smooth_iterations=iters)


def test_oracle_single_sprite_depth_is_the_sphere_front():
    """CPU: one particle on the view axis; the centre pixel's depth is the
    distance to the particle minus its radius (the sprite is a sphere impostor)."""
    w = h = 33
    cam = render.make_camera((0.0, 0.0, 5.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), math.radians(30.0), w, h, 0.5,
                             smooth_iterations=0)
    z, th = RO.splat(cam, np.zeros((1, 3), np.float32), w, h)
    assert abs(z[16, 16] - 4.5) < 1e-3 and abs(th[16, 16] - 1.0) < 1e-3
    assert z[0, 0] == 0 and np.count_nonzero(z) == np.count_nonzero(th) > 20


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,iters", [(96, 72, 6), (64, 64, 60)])
def test_render_passes_match_oracle(w, h, iters):
    import torch
    pos = _blob()
    cam = _cam(w, h, iters)
    r = render.Renderer(w, h)
    d = torch.from_numpy(pos).cuda()
    r.frame(cam, positions=d, stride=3)
    want = RO.render(cam, pos, w, h)
    for name in ("depth_raw", "depth", "thickness", "normal", "room"):
        got = r.read(name)
        assert np.array_equal(got.view(np.uint32), want[name].view(np.uint32)), name
    got = r.read("color")
    assert np.count_nonzero(want["depth"]) > 200
    assert np.abs(got - want["color"]).max() <= 2e-5
    r.close()


@pytest.mark.gpu
def test_render_solver_state_equals_its_positions():
    """The image does not depend on particle order: rendering the solver's own
    state (cell order, float4) equals rendering its downloaded positions."""
    import torch
    from pbf_b200 import Solver
    sc = scenes.dam_break(12, (40, 20, 20), stable=True, iterations=2)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    s.upload(sc.pos, sc.vel)
    s.step(3)
    w, h = 80, 60
    cam = render.box_camera(sc.grid_space, w, h, 0.03, smooth_iterations=10)
    a = render.Renderer(w, h)
    a.frame(cam, solver=s)
    p, _ = s.download()
    b = render.Renderer(w, h)
    b.frame(cam, positions=torch.from_numpy(p).cuda(), stride=3)
    for name in ("depth", "thickness", "color"):
        assert np.array_equal(a.read(name), b.read(name)), name
    assert np.count_nonzero(a.read("depth")) > 50


@pytest.mark.gpu
def test_render_rejects_bad_arguments():
    from pbf_b200._lib import PBFError
    with pytest.raises(PBFError):
        render.Renderer(0, 10)
    r = render.Renderer(8, 8)
    cam = _cam(8, 8)
    cam.smooth_iterations = -1
    import torch
    with pytest.raises(PBFError):
        r.frame(cam, positions=torch.zeros((4, 3), device="cuda"), stride=3)


@pytest.mark.gpu
def test_render_known_answers_on_the_gpu():
    """The closed forms of tests/test_render_pins.py straight through the CUDA
    passes: two overlapping sprites (sphere fronts under the depth test, chords
    summed) and the room seen head-on from inside."""
    import torch
    from test_render_pins import _room_centre, _sphere_profile, _sprite_camera
    w = h = 129
    dist = 5.0
    cam = _sprite_camera(w, h, dist, 0.5)
    second = (0.6, 0.1, -0.3)
    pos = np.array([[0.0, 0.0, 0.0], second], np.float32)
    r = render.Renderer(w, h)
    r.frame(cam, positions=torch.from_numpy(pos).cuda(), stride=3)
    z, th = r.read("depth_raw"), r.read("thickness")
    r.close()
    c1, q1, d1, t1 = _sphere_profile(cam, w, h)
    c2, q2, d2, t2 = _sphere_profile(cam, w, h, second)
    inside = ((q1 < 0.99) | (q1 > 1.01)) & ((q2 < 0.99) | (q2 > 1.01))
    want_z = np.where(c1 & c2, np.minimum(d1, d2), np.where(c1, d1, np.where(c2, d2, 0.0)))
    want_t = np.where(c1, t1, 0.0) + np.where(c2, t2, 0.0)
    assert np.abs(z[inside] - want_z[inside]).max() <= 2e-6 * dist
    assert np.abs(th[inside] - want_t[inside]).max() <= 1e-5
    # the room: the back wall head-on, lit by the light above the room's centre
    w = h = 33
    cam = render.make_camera((0.0, 25.0, 20.0), (0.0, 25.0, -30.0), (0, 1, 0), math.radians(40.0), w, h, 0.1)
    r = render.Renderer(w, h)
    r.frame(cam, positions=torch.zeros((1, 3), device="cuda") + 1000.0, stride=3)  # no particle in view
    got = r.read("room")[h // 2, w // 2]
    r.close()
    assert np.array_equal(got, _room_centre((0.0, 25.0, 20.0), (0.0, 25.0, -30.0), (0, 1, 0)))
    assert np.all(got[:3] == np.float32(200.0 / 255.0))
