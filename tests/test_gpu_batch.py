"""Batched scenes (GPU tests): each scene of a batch advances exactly as it would
alone. One launch per phase covers every scene and one scan over the
concatenated cell keys sorts them all, yet scene s's slot range holds, bit for
bit, what the oracle computes for scene s by itself."""
import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import BatchSolver, Solver, scenes

pytestmark = pytest.mark.gpu


def run_batch(scs, substeps, **ext):
    para, descs, ov, pos, vel = scenes.batch_inputs(scs)
    ov.update(ext)
    b = BatchSolver(para, descs, scenes.default_ext(**ov))
    b.upload(pos, vel)
    b.step(substeps)
    return b


def check_scene_vs_oracle(b, i, sc, substeps, **ext):
    lay = b.scene_layout(i)
    lo, hi = lay["pbase"], lay["pbase"] + lay["pcount"]
    orc = O.Oracle(O.params_for_scene(sc, ext), sc.pos, sc.vel)
    orc.substep(substeps)
    perm = b.fetch("perm")[lo:hi] - lo
    assert np.array_equal(perm, orc.get("perm")), f"scene {i}: perm"
    for name in ("x", "v"):
        got = b.fetch(name)[lo:hi, :3]
        want = orc.get(name).astype(np.float32)
        bad = int((got.view(np.uint32) != want.view(np.uint32)).sum())
        assert bad == 0, f"scene {i}: {name} differs in {bad} values"


def test_batch_bitexact_vs_each_scene_alone():
    scs = scenes.config2(seed=3, n_scenes=6, lo=300, hi=3000)
    b = run_batch(scs, 3)
    assert b.nscenes == 6
    for i, sc in enumerate(scs):
        check_scene_vs_oracle(b, i, sc, 3)


def test_batch_with_sphere_walls_and_out_of_grid_scene():
    scs = scenes.config2(seed=5, n_scenes=3, lo=500, hi=2000)
    # scene 1: a grid smaller than its box (out-of-grid bin in the middle of the key space)
    d = scs[1].ext_overrides["grid_dims"]
    scs[1].ext_overrides["grid_dims"] = [max(2, d[0] // 2), d[1], d[2]]
    # scene 2: a sphere obstacle in its box and fast particles
    box = scs[2].grid_space
    scs[2].ext_overrides["sphere"] = (0.5 * box[3], 0.2, 0.5 * box[5], 0.15)
    rng = np.random.RandomState(9)
    scs[0].vel = rng.uniform(-30, 30, size=scs[0].pos.shape).astype(np.float32)
    b = run_batch(scs, 2)
    for i, sc in enumerate(scs):
        check_scene_vs_oracle(b, i, sc, 2)


def test_cell_scale_half_widens_stencil_bitexact():
    """Cells of h/2 with a 5x5x5 stencil find the same neighbours (in the
    oracle's matching order)."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, grid_dims=(80, 40, 40))
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(cell_scale=0.5))
    s.upload(sc.pos, sc.vel)
    s.step(2)
    orc = O.Oracle(O.params_for_scene(sc, {"cell_scale": 0.5}), sc.pos, sc.vel)
    orc.substep(2)
    assert np.array_equal(s.fetch("perm"), orc.get("perm"))
    for name in ("x", "v"):
        got = s.fetch(name)[:, :3]
        assert np.array_equal(got.view(np.uint32), orc.get(name).astype(np.float32).view(np.uint32)), name
    # the neighbour sets equal those of the default 27-cell stencil
    s1 = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(grid_dims=[40, 20, 20], debug=1))
    s2 = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(cell_scale=0.5, debug=1))
    for t in (s1, s2):
        t.upload(sc.pos, sc.vel)
        t.build_grid()
    p1, p2 = s1.fetch("perm"), s2.fetch("perm")
    sets1 = {int(p1[k]): sorted(int(p1[j]) for j in l) for k, l in enumerate(s1.neighbor_lists())}
    sets2 = {int(p2[k]): sorted(int(p2[j]) for j in l) for k, l in enumerate(s2.neighbor_lists())}
    assert sets1 == sets2


def test_batch_stats_and_density_error():
    scs = scenes.config2(seed=1, n_scenes=4, lo=1000, hi=4000)
    b = run_batch(scs, 4, measure_error=1)
    st = b.stats()
    assert st["error_bits"] == 0
    pos, _ = b.download()
    worst = 0.0
    off = 0
    for sc in scs:
        mx, _ = O.density_error(pos[off:off + sc.n], float(sc.para.h), float(sc.para.restRho))
        worst = max(worst, mx)
        off += sc.n
    assert abs(st["max_density_error"] - worst) <= 1e-4


@pytest.mark.parametrize("lanes,cell_scale", [(2, 1.0), (1, 0.5), (4, 0.5)])
def test_persistent_passes_bitexact(lanes, cell_scale):
    """Each neighbour pass as one persistent launch (the resident blocks stride
    over every scene's tiles of slots) gives the oracle's results bit for bit,
    like the one-block-per-tile launch, in the adaptive loop too."""
    scs = scenes.config2(seed=7, n_scenes=5, lo=800, hi=5000)
    for sc in scs:
        sc.ext_overrides["grid_dims"] = [int(round(d / cell_scale)) for d in sc.ext_overrides["grid_dims"]]
    ext = dict(persistent=1, pair_lanes=lanes, cell_scale=cell_scale, block_size=128)
    b = run_batch(scs, 3, **ext)
    for i, sc in enumerate(scs):
        check_scene_vs_oracle(b, i, sc, 3, pair_lanes=lanes, cell_scale=cell_scale)
    ad = run_batch(scs, 2, adaptive=1, density_tol=0.02, max_iterations=8, **ext)
    plain = run_batch(scs, 2, adaptive=1, density_tol=0.02, max_iterations=8, pair_lanes=lanes,
                      cell_scale=cell_scale, block_size=128)
    assert ad.stats()["total_iterations"] == plain.stats()["total_iterations"]
    for name in ("x", "v"):
        assert np.array_equal(ad.fetch(name).view(np.uint32), plain.fetch(name).view(np.uint32)), name
