"""Parity at the sizes the benchmark runs (GPU tests), bit for bit against the
oracle through the C ABI.

* the 262,144-particle dam break with the launch settings the benchmark's
  autotuner chooses between (cells of h and of h/2 with the 5^3 stencil, two
  pair lanes, 256 threads): every intermediate of two substeps from the initial
  lattice, and a substep from a developed state (40 substeps in, where the
  column has started to collapse);
* the full 64-scene batch (1,390,357 particles; counts log-uniform in
  [4,096, 65,536]) against each scene run alone by the oracle; above 2^20
  particles the hash and scatter take four slots per thread;
* one substep of the 4,718,592-particle double dam break with the sphere
  batched with 8 scenes of 65,536 particles: over 2^22 cell keys, so the scan
  runs its tiles of 16,384 counts.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import BatchSolver, Solver, autotune, scenes

from test_gpu_parity import assert_substep_bitexact

pytestmark = pytest.mark.gpu


def launch_ext(sc, cell_scale):
    return {"cell_scale": cell_scale, "grid_dims": autotune.dims_for_scale(sc.ext_overrides["grid_dims"], cell_scale),
            "block_size": 256, "pair_lanes": 2}


@pytest.mark.parametrize("cell_scale", [0.5, 1.0])
def test_config1_full_size_bitexact(cell_scale):
    sc = scenes.config1()
    assert sc.n == 262144
    ext = launch_ext(sc, cell_scale)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(debug=1, **ext))
    s.upload(sc.pos, sc.vel)
    orc = O.Oracle(O.params_for_scene(sc, ext), sc.pos, sc.vel)
    for _ in range(2):
        s.step(1)
        orc.substep()
        assert_substep_bitexact(s, orc)
    s.close()
    orc.close()


def test_config1_developed_state_bitexact():
    sc = scenes.config1()
    ext = launch_ext(sc, 0.5)
    run = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(**ext))
    run.upload(sc.pos, sc.vel)
    run.step(40)
    pos, vel = run.download()
    run.close()
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(debug=1, **ext))
    s.upload(pos, vel)
    orc = O.Oracle(O.params_for_scene(sc, ext), pos, vel)
    s.step(1)
    orc.substep()
    assert_substep_bitexact(s, orc)
    assert np.abs(vel).max() > 0.5  # the column is moving
    s.close()
    orc.close()


def run_batch(scs, substeps, cell_scale):
    para, descs, ov, pos, vel = scenes.batch_inputs(scs)
    for d in descs:
        d["grid_dims"] = autotune.dims_for_scale(d["grid_dims"], cell_scale)
    ov.update(cell_scale=cell_scale, block_size=256, pair_lanes=2)
    b = BatchSolver(para, descs, scenes.default_ext(**ov))
    b.upload(pos, vel)
    b.step(substeps)
    return b


def check_scenes(b, scs, substeps, cell_scale):
    perm_all = b.fetch("perm")
    x_all = b.fetch("x")
    v_all = b.fetch("v")
    for i, sc in enumerate(scs):
        lay = b.scene_layout(i)
        lo, hi = lay["pbase"], lay["pbase"] + lay["pcount"]
        ext = {"cell_scale": cell_scale,
               "grid_dims": autotune.dims_for_scale(sc.ext_overrides["grid_dims"], cell_scale)}
        orc = O.Oracle(O.params_for_scene(sc, ext), sc.pos, sc.vel)
        orc.substep(substeps)
        assert np.array_equal(perm_all[lo:hi] - lo, orc.get("perm")), f"scene {i}: perm"
        for name, got in (("x", x_all), ("v", v_all)):
            want = orc.get(name).astype(np.float32)
            bad = int((got[lo:hi, :3].view(np.uint32) != want.view(np.uint32)).sum())
            assert bad == 0, f"scene {i}: {name} differs in {bad} values"
        orc.close()


@pytest.mark.parametrize("cell_scale", [1.0, 0.5])
def test_config2_full_batch_bitexact(cell_scale):
    scs = scenes.config2(seed=0)
    assert len(scs) == 64 and sum(s.n for s in scs) > (1 << 20)
    b = run_batch(scs, 1, cell_scale)
    assert b.stats()["error_bits"] == 0
    check_scenes(b, scs, 1, cell_scale)
    b.close()


def test_config4_one_substep_bitexact():
    scs = scenes.config4(seed=0)
    assert sum(s.n for s in scs) == 4718592
    b = run_batch(scs, 1, 1.0)
    assert b.stats()["error_bits"] == 0
    nkeys = sum(b.scene_layout(i)["ncells"] + 1 for i in range(b.nscenes))
    assert nkeys > (1 << 22)
    check_scenes(b, scs, 1, 1.0)
    b.close()
