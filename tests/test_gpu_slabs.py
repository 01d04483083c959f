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
