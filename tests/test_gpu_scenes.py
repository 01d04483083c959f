"""Scene generators (GPU tests): the reference app's five initial conditions
(src/renderapp.cpp:137-234, h = 1, rho0 = 6, gravity -49) and the batched
workloads run through the solver, stay finite and stay inside their walls."""
import numpy as np
import pytest

from pbf_b200 import BatchSolver, Solver, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("idx", [1, 2, 3, 4, 5])
def test_reference_app_scene(idx):
    sc = scenes.reference_app_scene(idx, dims=(24, 24, 24))
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    s.upload(sc.pos, sc.vel)
    s.step(5)
    st = s.stats()
    assert st["error_bits"] == 0
    pos, vel = s.download()
    assert np.isfinite(pos).all() and np.isfinite(vel).all()
    lo, hi = np.array(sc.boundary[:3]), np.array(sc.boundary[3:])
    assert (pos >= lo - 1e-4).all() and (pos <= hi + 1e-4).all()


def test_double_dam_break_with_sphere_small():
    scs = scenes.config4(block=20, small=2000, n_small=2, iterations=3)
    para, descs, ov, pos, vel = scenes.batch_inputs(scs)
    b = BatchSolver(para, descs, scenes.default_ext(**ov))
    b.upload(pos, vel)
    b.step(10)
    assert b.stats()["error_bits"] == 0
    x, _ = b.download()
    big = scs[0]
    c = np.array(big.ext_overrides["sphere"][:3])
    r = big.ext_overrides["sphere"][3]
    d = np.linalg.norm(x[: big.n] - c, axis=1)
    assert d.min() >= r * (1 - 1e-5)
