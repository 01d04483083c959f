"""The oracle's GPU formulation against the reference's own CUDA solver (CPU test).

tests/golden/refgpu_dam16_it{1,4}.npz hold the outputs of kernels/cudaPBF.cu +
kernels/cudaPBFSolver.cu, built unmodified and run on a B200 by
tests/golden/make_golden.py gpu, for the seeded 16^3 dam break with the
reference's literal parameters (gravity -49 as in kernels/cudaPBFSolver.cu:9).

* cell ranges, neighbour counts and neighbour sets depend only on predicted
  positions and must match exactly;
* the reference's in-cell order is racy (atomicSub, kernels/cudaPBFSolver.cu:119),
  so the sorted ids are compared as per-cell sets;
* floating-point fields are compared away from the walls: the wall clamp hashes
  positions through sinf(...) * 43758.5453 (cuh:116-119), which turns an ulp of
  difference into a different offset, so clamped particles and their neighbours
  differ by design. With one iteration every interior field agrees to 1e-5 of
  its scale (x 1e-7, lambda 4e-7, dp 2e-6, v 3e-6, vorticity 8e-6; the
  prediction rounds once per update, as the reference's build contracts it). With four iterations at these (diverging) parameters the interior
  is reached by the wall differences, so only the integer stages are compared.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def run_oracle(iterations):
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    sc.para.iterations = iterations
    op = O.params_from(sc.para, sc.grid_space, sc.boundary, gravity=(0.0, -49.0, 0.0), dims=(64, 64, 64),
                       formulation=0, arith=0, cell_order=0, reorder=0)
    orc = O.Oracle(op, sc.pos, sc.vel)
    orc.substep()
    return sc, orc


@pytest.mark.parametrize("iterations", [1, 4])
def test_integer_stages_match_reference_cuda(iterations):
    g = np.load(os.path.join(GOLDEN, f"refgpu_dam16_it{iterations}.npz"))
    sc, orc = run_oracle(iterations)
    assert np.array_equal(g["pos_in"], sc.pos)
    st, en = orc.get("start"), orc.get("end")
    cells = g["grid_cells"]
    assert np.array_equal(np.nonzero(en > st)[0], cells)
    assert np.array_equal(st[cells], g["grid_start"]) and np.array_equal(en[cells], g["grid_end"])
    sorted_ref, sorted_orc = g["sorted"], orc.get("sorted")
    for c, s, e in zip(cells, g["grid_start"], g["grid_end"]):
        assert set(sorted_ref[s:e]) == set(sorted_orc[s:e]), c
    n = sc.n
    nb, cnt = g["nbr"], g["nbr"][:, 63]
    on, oc = orc.get("nbr").reshape(n, 63), orc.get("ncnt")
    assert np.array_equal(cnt, oc)
    for i in range(n):
        assert set(nb[i, :cnt[i]]) == set(on[i, :oc[i]]), i


def test_interior_fields_match_reference_cuda_one_iteration():
    g = np.load(os.path.join(GOLDEN, "refgpu_dam16_it1.npz"))
    sc, orc = run_oracle(1)
    x = orc.get("x")
    lo, hi = np.array(sc.boundary[:3]), np.array(sc.boundary[3:])
    dist = np.minimum(x - lo, hi - x).min(1)
    h = float(sc.para.h)
    assert np.array_equal(g["xold"].astype(np.float64), orc.get("xold"))
    for name, margin in (("x", 2 * h), ("v", 2 * h), ("lambda", 2 * h), ("dp", 2 * h), ("curl", 2 * h),
                         ("visc", 2 * h), ("vort", 3 * h)):
        ref = g[name].astype(np.float64)
        got = orc.get(name)
        m = dist > margin
        assert m.sum() > 800
        d = np.abs(ref - got)
        d = d.max(1) if d.ndim > 1 else d
        assert d[m].max() <= 1e-5 * np.abs(ref).max(), (name, d[m].max() / np.abs(ref).max())
