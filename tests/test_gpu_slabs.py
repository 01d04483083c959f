"""Slab decomposition on the GPU (pbf_b200/slabs.py): the slabs of one scene run
as separate CUDA solvers on one device (the exchange a tensor copy) and match
the single-domain solver bit for bit, positions and velocities, over several
substeps while particles cross the slab faces."""
import numpy as np
import pytest
import torch

from pbf_b200 import Solver, slabs

from test_slabs_cpu import slab_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nslabs,iterations,cell_scale", [(2, 2, 1.0), (3, 2, 1.0), (2, 4, 1.0), (2, 2, 0.5)])
def test_slabs_match_single_domain_bitexact(nslabs, iterations, cell_scale):
    sc = slab_scene(iterations=iterations)
    dims = [int(round(d / cell_scale)) for d in sc.ext_overrides["grid_dims"]]
    ext = sc.ext(cell_scale=cell_scale, grid_dims=dims)
    steps = 6
    ref = Solver(sc.para, sc.grid_space, sc.boundary, ext)
    ref.upload(sc.pos, sc.vel)
    ref.step(steps)
    want_x, want_v = ref.download()
    geom = slabs.SlabGeometry(sc.para, sc.grid_space, ext, nslabs)
    engines = [slabs.CudaEngine(sc.para, sc.grid_space, sc.boundary, ext, sc.n) for _ in range(nslabs)]
    group = slabs.SlabGroup(geom, engines)
    group.load(torch.from_numpy(sc.pos).cuda(), torch.from_numpy(sc.vel).cuda())
    for _ in range(steps):
        group.step()
        assert sum(len(s.own) for s in group.ranks) == sc.n
    assert min(len(s.own) for s in group.ranks) > 0
    x, v = group.gather()
    assert np.array_equal(x.cpu().numpy().view(np.uint32), want_x.view(np.uint32))
    assert np.array_equal(v.cpu().numpy().view(np.uint32), want_v.view(np.uint32))


def test_resize_and_sorted_state_errors():
    from pbf_b200 import BatchSolver, scenes
    from pbf_b200._lib import PBF_ERR_INVALID, PBF_ERR_STATE, PBFError
    sc = slab_scene()
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    for bad in (0, sc.n + 1):
        with pytest.raises(PBFError) as e:
            s.resize(bad)
        assert e.value.code == PBF_ERR_INVALID
    s.upload(sc.pos, sc.vel)
    out = torch.empty((sc.n, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(PBFError) as e:
        s.download_sorted_device(pos=out)  # no substep since the upload
    assert e.value.code == PBF_ERR_STATE
    s.resize(100)
    with pytest.raises(PBFError) as e:
        s.step(1)  # a resize needs a new upload
    assert e.value.code == PBF_ERR_STATE
    s.upload(sc.pos[:100], sc.vel[:100])
    s.step(1)
    ids = torch.empty(100, dtype=torch.int32, device="cuda")
    key = torch.empty(100, dtype=torch.int32, device="cuda")
    rank = torch.empty(100, dtype=torch.int32, device="cuda")
    s.download_sorted_device(ids=ids, key=key, rank=rank)
    assert sorted(ids.cpu().tolist()) == list(range(100))
    k, r = key.cpu().numpy().astype(np.int64), rank.cpu().numpy()
    assert np.all(np.diff(k) >= 0)  # slot order is cell order
    first = np.r_[True, k[1:] != k[:-1]]
    assert np.all(r[first] == 0) and np.all(r[~first] == r[np.flatnonzero(~first) - 1] + 1)
    para, descs, ov, pos, vel = scenes.batch_inputs([scenes.dam_break(4), scenes.dam_break(4)])
    b = BatchSolver(para, descs, scenes.default_ext(**ov))
    with pytest.raises(PBFError) as e:
        b.resize(10)
    assert e.value.code == PBF_ERR_INVALID


def test_step_host_argument_checks():
    sc = slab_scene()
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    good = np.zeros((sc.n, 3), np.float32)
    with pytest.raises(ValueError):
        s.step_host(good[:-1], good, good)
    with pytest.raises(ValueError):
        s.step_host(good, good.astype(np.float64), good)
    ro = good.copy()
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        s.step_host(good, good, ro)
