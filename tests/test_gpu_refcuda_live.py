"""The library against the reference's own CUDA solver, both run live on the GPU
(oracle/_ref/libpbfref_gpu.so: kernels/cudaPBF.cu and kernels/cudaPBFSolver.cu
built unmodified), on the reference app's scenes at the reference's default size
(64^3 = 262,144 particles, src/renderapp.cpp:137-234: h = 1, rho0 = 6, eps = 1,
k = 0.01, 4 Jacobi iterations, gravity -49, 64^3 grid).

The reference is not deterministic: its counting sort fills each cell with
atomicSub (kernels/cudaPBFSolver.cu:119), so the neighbour lists come in a
different order on every run and the FP32 sums round differently. The test
therefore runs the reference twice on the same input and requires the library
to agree with the first run as closely as the second run does (interior
particles, every field), with the neighbour counts equal everywhere away from
the walls. x and v agree to 1e-5 of their scale; lambda and dp depart by up to
3e-5 in both comparisons, the rounding spread of the reference itself.

Particles the wall clamp moves differ by design: the reference hashes their
offset through sinf (kernels/cudaPBFSolver.cuh:116-119), the library through a
double-precision sine of its own, and the offset is a fractional part of
sin(...) * 43758.5453, so one ulp of the sine moves it anywhere in
[0, RANDOM_OFFSET_COEFF). With one clamped axis the clamped position differs by
at most 0.01 (include/solverBase.h:5); four Jacobi iterations spread that into
the particle's neighbours, bounded here at 4 x 0.01 (measured on the floor
layer of scene 1 moving down: at most 0.0098 for the 4,096 clamped particles
and 0.031 for any particle).

The library's prediction v += dt g, x += dt v rounds each update once (a fused
multiply-add), as the reference's build of those lines does; with two
roundings, pairs at exactly h left the neighbour list in one solver and not the
other, and such a pair acts for every later Jacobi iteration.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import Solver, scenes

pytestmark = pytest.mark.gpu

RANDOM_OFFSET_COEFF = 0.01


def run_ours(sc):
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(debug=1))
    s.upload(sc.pos, sc.vel)
    s.step(1)
    perm = s.fetch("perm")

    def orig(a):
        out = np.empty_like(a)
        out[perm] = a
        return out

    out = {"x": orig(s.fetch("x")[:, :3]), "v": orig(s.fetch("v")[:, :3]), "lambda": orig(s.fetch("xl")[:, 3]),
           "dp": orig(s.fetch("dp")[:, :3]), "ncnt": orig(s.fetch("ncnt"))}
    s.close()
    return out


def residual(a, b, mask):
    """max |a - b| over the masked particles, relative to max |b| there."""
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    bb = np.abs(b.astype(np.float64))
    if d.ndim > 1:
        d, bb = d.max(1), bb.max(1)
    return float(d[mask].max() / bb[mask].max())


def scene(idx, vdown=0.0):
    sc = scenes.reference_app_scene(idx)
    if vdown:
        sc.vel = np.tile(np.float32([0.0, -vdown, 0.0]), (sc.n, 1))
    return sc


def interior(sc, x_end, margin_h):
    lo, hi = np.array(sc.boundary[:3]), np.array(sc.boundary[3:])
    h = float(sc.para.h)
    d0 = np.minimum(sc.pos - lo, hi - sc.pos).min(1)
    d1 = np.minimum(x_end - lo, hi - x_end).min(1)
    return np.minimum(d0, d1) > margin_h * h


@pytest.mark.skipif(not O.refgpu_available(), reason="reference CUDA solver not built (needs the reference sources)")
@pytest.mark.parametrize("idx,vdown", [(1, 0.0), (4, 0.0), (5, 0.0), (1, 20.0)])
def test_interior_within_the_reference_own_spread(idx, vdown):
    sc = scene(idx, vdown)
    assert sc.n == 262144
    ra = O.refgpu_run(sc.para, sc.grid_space, sc.boundary, sc.pos, sc.vel, substeps=1)
    rb = O.refgpu_run(sc.para, sc.grid_space, sc.boundary, sc.pos, sc.vel, substeps=1)
    ours = run_ours(sc)
    inner = interior(sc, ra["x"], 5)
    assert inner.sum() > 150000
    # neighbour counts: the reference's own are run-independent; ours equal them
    assert np.array_equal(ra["nbr"][:, 63], rb["nbr"][:, 63])
    assert np.array_equal(ours["ncnt"][inner], ra["nbr"][inner, 63])
    report = {}
    for name in ("x", "v", "lambda", "dp"):
        own = residual(rb[name], ra[name], inner)
        got = residual(ours[name], ra[name], inner)
        report[name] = (got, own)
        assert got <= 2.0 * own + 1e-6, (name, got, own)
    assert report["x"][0] <= 1e-5 and report["v"][0] <= 1e-5, report
    print(f"scene {idx} vdown {vdown}: (ours, reference run 2) vs reference run 1:", report)


@pytest.mark.skipif(not O.refgpu_available(), reason="reference CUDA solver not built (needs the reference sources)")
def test_wall_clamped_particles_within_the_offset_bound():
    sc = scene(1, 20.0)  # the bottom layers reach the floor in the first prediction
    ra = O.refgpu_run(sc.para, sc.grid_space, sc.boundary, sc.pos, sc.vel, substeps=1)
    ours = run_ours(sc)
    dt = np.float32(sc.para.dt)
    v1 = sc.vel + dt * np.float32([0.0, -49.0, 0.0])
    xp = sc.pos + dt * v1
    lo, hi = np.float32(sc.boundary[:3]), np.float32(sc.boundary[3:])
    clamped = ((xp < lo) | (xp > hi)).any(1)
    assert clamped.sum() >= 4096  # the whole bottom layer of the 64^3 lattice
    d = np.abs(ours["x"].astype(np.float64) - ra["x"].astype(np.float64)).max(1)
    # the clamped particles themselves: within the offset range (measured 0.0098)
    assert d[clamped].max() <= 2 * RANDOM_OFFSET_COEFF, d[clamped].max()
    assert np.quantile(d[clamped], 0.99) <= RANDOM_OFFSET_COEFF
    # their neighbours, through four Jacobi iterations (measured 0.031)
    assert d.max() <= 4 * RANDOM_OFFSET_COEFF, d.max()
    # every particle stays inside the walls in both
    for x in (ours["x"], ra["x"]):
        assert (x >= lo - 1e-5).all() and (x <= hi + 1e-5).all()
