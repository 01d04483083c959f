"""The oracle is pinned against the reference itself (CPU tests).

* formulation 1 / reference arithmetic vs the reference's own CPU solver
  (src/solver.cpp + include/solver.h compiled as-is into oracle/_ref): every
  field bit-exact, over several substeps and iteration counts;
* the same against the committed fixture made from that solver
  (tests/golden/make_golden.py), so the pin holds where the reference
  sources are absent;
* the deterministic sine against the true sine;
* the FP64 density-error oracle against a brute-force evaluation.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

needs_refcpu = pytest.mark.skipif(not O.refcpu_available(), reason="reference CPU solver not built here")


def _cpu_form_params(sc, iterations, dims=(64, 64, 64)):
    return O.params_from(sc.para, sc.grid_space, sc.boundary, gravity=(0.0, -9.8, 0.0), dims=dims, formulation=1,
                         arith=0, cell_order=1, reorder=0, wall_jitter=0.02, iterations=iterations)


def _compare_all(ref, orc, p_ref, v_ref):
    for name in ("start", "end", "sorted", "cell", "ncnt", "nbr"):
        a, b = ref.get(name), orc.get(name)
        if name == "sorted":
            # only the in-grid prefix of gridParticlesID is defined in the reference
            k = int(ref.get("end")[-1]) if ref.ncells else 0
            inside = int(np.count_nonzero(ref.get("cell") >= 0))
            a, b = a[:inside], b[:inside]
        assert np.array_equal(a, b), name
    for name, ra in (("lambda", ref.get("lambda")), ("dp", ref.get("dp")), ("curl", ref.get("curl")),
                     ("vort", ref.get("vort")), ("visc", ref.get("visc")), ("xold", ref.get("xold")),
                     ("x", p_ref), ("v", v_ref)):
        ob = orc.get(name).astype(np.float32)
        assert np.array_equal(np.asarray(ra, np.float32).view(np.uint32), ob.view(np.uint32)), name


@needs_refcpu
@pytest.mark.parametrize("iterations,substeps", [(1, 1), (4, 1), (4, 3), (0, 1)])
def test_oracle_bitexact_vs_reference_cpu_solver(iterations, substeps):
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    sc.para.iterations = iterations
    ref = O.RefCpu(sc.para, sc.grid_space)
    p, v = ref.solve(sc.pos, sc.vel, substeps=substeps)
    orc = O.Oracle(_cpu_form_params(sc, iterations), sc.pos, sc.vel)
    orc.substep(substeps)
    _compare_all(ref, orc, p, v)


@needs_refcpu
def test_oracle_bitexact_vs_reference_cpu_walls_and_outside_grid():
    """Particles thrown at every wall (the clamp and its hashed offset run on
    most of them) with a grid smaller than the box (out-of-grid particles get
    no cell, kernels/cudaPBFSolver.cuh:163-181)."""
    sc = scenes.dam_break(12, (20, 10, 10), stable=False)
    rng = np.random.RandomState(7)
    vel = rng.uniform(-40, 40, size=sc.pos.shape).astype(np.float32)
    sc.para.iterations = 2
    dims = (16, 8, 12)
    ref = O.RefCpu(sc.para, sc.grid_space, dims=dims)
    p, v = ref.solve(sc.pos, vel, substeps=2)
    orc = O.Oracle(_cpu_form_params(sc, 2, dims=dims), sc.pos, vel)
    orc.substep(2)
    assert np.count_nonzero(orc.get("cell") < 0) > 0
    _compare_all(ref, orc, p, v)


@needs_refcpu
def test_oracle_grid_build_bitexact_vs_reference_buildNeiborhood():
    """buildNeiborhood (src/solver.cpp:3-58) on given positions."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    ref = O.RefCpu(sc.para, sc.grid_space)
    ref.build(sc.pos)
    orc = O.Oracle(_cpu_form_params(sc, 1), sc.pos, sc.vel)
    orc.build_only()
    for name in ("start", "end", "sorted", "cell", "ncnt", "nbr"):
        assert np.array_equal(ref.get(name), orc.get(name)), name


def test_oracle_vs_golden_reference_cpu_fixture():
    g = np.load(os.path.join(GOLDEN, "refcpu_dam16.npz"))
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    assert np.array_equal(sc.pos, g["pos_in"])
    sc.para.iterations = int(g["iterations"])
    orc = O.Oracle(_cpu_form_params(sc, int(g["iterations"])), sc.pos, sc.vel)
    orc.substep(int(g["substeps"]))
    for name in ("x", "v", "lambda", "dp", "curl", "vort", "visc"):
        assert np.array_equal(g[name].view(np.uint32), orc.get(name).astype(np.float32).view(np.uint32)), name
    for name in ("start", "end", "ncnt"):
        assert np.array_equal(g[name], orc.get(name)), name


def test_det_sin_within_one_ulp():
    rng = np.random.RandomState(3)
    args = np.concatenate([rng.uniform(-4000, 4000, 20000), rng.uniform(-3.2, 3.2, 5000),
                           np.array([0.0, 1e-30, -1e-30, math.pi / 2, math.pi, 1e5])]).astype(np.float32)
    for a in args:
        got = np.float32(O.det_sin(float(a)))
        exact = math.sin(float(a))
        ulp = np.spacing(np.float32(abs(exact))) if exact != 0 else np.float32(1e-45)
        assert abs(float(got) - exact) <= float(ulp), (a, got, exact)


def test_density_error_oracle_bruteforce():
    rng = np.random.RandomState(5)
    pos = rng.uniform(0, 0.4, size=(600, 3)).astype(np.float32)
    h, rho0 = float(np.float32(0.1)), 200.0  # the oracle takes h as a float
    mx, mean, err = O.density_error(pos, h, rho0, per_particle=True)
    p = pos.astype(np.float64)
    d2 = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    w = np.where(d2 <= h * h, 315.0 / (64.0 * math.pi * h ** 9) * (h * h - np.minimum(d2, h * h)) ** 3, 0.0)
    rho = w.sum(1)
    e = np.maximum(rho / rho0 - 1.0, 0.0)
    assert np.allclose(err, e, rtol=1e-12, atol=1e-12)
    assert math.isclose(mx, e.max(), rel_tol=1e-12) and math.isclose(mean, e.mean(), rel_tol=1e-12)


def test_oracle_product_vs_reference_arithmetic_close():
    """The product arithmetic departs from the reference arithmetic only in
    rounding (cubes vs powf, fused sums, one division in the gradient): on the
    interior (no wall clamp) one substep agrees to ~1e-6 relative."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True)
    base = dict(gravity=(0.0, -9.8, 0.0), dims=(40, 20, 20), formulation=0, cell_order=0, reorder=0,
                flags=sc.ext_overrides["flags"], scorr_scale=sc.ext_overrides["scorr_scale"], iterations=4)
    a = O.Oracle(O.params_from(sc.para, sc.grid_space, sc.boundary, arith=0, **base), sc.pos, sc.vel)
    b = O.Oracle(O.params_from(sc.para, sc.grid_space, sc.boundary, arith=1, **base), sc.pos, sc.vel)
    a.substep()
    b.substep()
    lam_a, lam_b = a.get("lambda"), b.get("lambda")
    # C = rho/rho0 - 1 cancels; the size of the terms behind lambda is (rho/rho0)/eps
    scale = a.get("rho").max() / float(sc.para.restRho) / float(sc.para.epsilon)
    assert np.abs(lam_a - lam_b).max() <= 1e-5 * scale
    xa, xb = a.get("x"), b.get("x")
    interior = np.all((xa > np.array(sc.boundary[:3]) + 0.02) & (xa < np.array(sc.boundary[3:]) - 0.02), axis=1)
    assert interior.mean() > 0.5
    assert np.abs(xa[interior] - xb[interior]).max() <= 1e-5 * np.abs(xa).max()


@pytest.mark.parametrize("lanes", [2, 4, 8])
def test_oracle_pair_lane_sums_depart_only_by_rounding(lanes):
    """Splitting a neighbour sum over pair lanes changes only the FP32 summation
    order: against one sequential sum, lambda and positions agree to rounding."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True)
    base = dict(gravity=(0.0, -9.8, 0.0), dims=(40, 20, 20), formulation=0, arith=1,
                flags=sc.ext_overrides["flags"], scorr_scale=sc.ext_overrides["scorr_scale"], iterations=4)
    a = O.Oracle(O.params_from(sc.para, sc.grid_space, sc.boundary, lanes=1, **base), sc.pos, sc.vel)
    b = O.Oracle(O.params_from(sc.para, sc.grid_space, sc.boundary, lanes=lanes, **base), sc.pos, sc.vel)
    a.substep()
    b.substep()
    assert np.array_equal(a.get("nbr"), b.get("nbr"))
    lam_a, lam_b = a.get("lambda"), b.get("lambda")
    assert not np.array_equal(lam_a, lam_b)  # the order does change the rounding
    scale = a.get("rho").max() / float(sc.para.restRho) / float(sc.para.epsilon)
    assert np.abs(lam_a - lam_b).max() <= 1e-5 * scale
    assert np.abs(a.get("x") - b.get("x")).max() <= 1e-5 * np.abs(a.get("x")).max()


def test_soft_rsqrt_within_two_ulp():
    """The product arithmetic's reciprocal square root (bit-level estimate plus
    three Newton steps) against double precision, over the |r|^2 range of the
    neighbour sums and a wide sweep of binades."""
    rng = np.random.RandomState(5)
    xs = np.concatenate([rng.uniform(1e-6, 1.0, 4000), 2.0 ** rng.uniform(-60, 60, 4000)]).astype(np.float32)
    worst = 0.0
    for x in xs:
        y = np.float32(O.rsqrt(float(x)))
        exact = 1.0 / math.sqrt(float(x))
        worst = max(worst, abs(float(y) - exact) / float(np.spacing(np.float32(exact))))
    assert worst <= 2.0, worst


def test_oracle_adaptive_substep_limits():
    """The adaptive substep at its two limits: a tolerance every state meets runs
    exactly the minimum count and equals the plain substep with that count; a
    zero tolerance runs to the cap. In between, the count lies between them and
    the lambda pass of the last correction measured an error above tolerance."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    prm = O.params_for_scene(sc)
    plain = O.Oracle(prm, sc.pos, sc.vel)
    loose = O.Oracle(prm, sc.pos, sc.vel)
    tight = O.Oracle(prm, sc.pos, sc.vel)
    mid = O.Oracle(prm, sc.pos, sc.vel)
    for _ in range(2):
        plain.substep()
        assert loose.substep_adaptive(1e30, 3, 12) == 3
        assert tight.substep_adaptive(0.0, 1, 5) == 5
        assert 1 <= mid.substep_adaptive(float(np.float32(0.003)), 1, 12) <= 12
    for name in ("x", "v", "curl", "vort"):  # (lambda differs: the adaptive loop measures once more)
        assert np.array_equal(plain.get(name), loose.get(name)), name
    assert not np.array_equal(plain.get("x"), tight.get("x"))
