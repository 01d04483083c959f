"""Slab decomposition of one scene (pbf_b200/slabs.py) on CPU: two gloo ranks,
each running its slab's substeps with the oracle (the CPU restatement, as the
checker's engine), against the oracle's single-domain run bit for bit. The
CUDA engine is compared the same way in test_gpu_slabs.py."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import oracle as O
from pbf_b200 import scenes, slabs


class OracleEngine:
    """One substep of a particle set with the oracle; the state in slot order."""

    def __init__(self, sc):
        self.prm = O.params_for_scene(sc)
        self.ncells = int(np.prod(sc.ext_overrides["grid_dims"]))

    def run(self, pos, vel):
        o = O.Oracle(self.prm, pos.numpy(), vel.numpy())
        o.substep()
        cell = o.get("cell")
        start = o.get("start")
        slot = np.arange(len(cell))
        key = np.where(cell < 0, self.ncells, cell)
        rank = slot - np.where(cell < 0, int(np.count_nonzero(cell >= 0)), start[np.maximum(cell, 0)])
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).astype(dt))  # noqa: E731
        return (t(o.get("x"), np.float32), t(o.get("v"), np.float32), t(o.get("perm"), np.int32), t(key, np.int32),
                t(rank, np.int32))


def slab_scene(iterations=2):
    """An 80 x 10 x 10 lattice at spacing h/2 from x = 6h in a 60h x 16h x 16h box:
    it spans both halves of the grid, each half holds particles the other's halo
    does not reach, and it breaks to the right."""
    sc = scenes.dam_break(4, (60, 16, 16), stable=True, iterations=iterations)
    rng = np.random.RandomState(3)
    h = float(sc.para.h)
    sc.pos = scenes.lattice_block((80, 10, 10), 0.5 * h, (6.0 * h, 0.5 * h, 0.5 * h), rng, 0.01 * h)
    sc.vel = np.zeros_like(sc.pos)
    sc.para.nParticles = sc.n
    return sc


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, steps, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sc = slab_scene()
    geom = slabs.SlabGeometry(sc.para, sc.grid_space, sc.ext(), world)
    slab = slabs.SlabRank(geom, rank, OracleEngine(sc))
    slab.load(torch.from_numpy(sc.pos), torch.from_numpy(sc.vel))
    comm = slabs.DistComm(rank, world, torch.device("cpu"))
    counts = []
    for _ in range(steps):
        comm.step(slab)
        counts.append(len(slab.own))
    pos, vel = comm.gather(slab)
    if rank == 0:
        q.put((pos.numpy(), vel.numpy(), counts))
    else:
        q.put((None, None, counts))
    dist.barrier()
    dist.destroy_process_group()


def test_geometry():
    sc = slab_scene(iterations=2)
    g = slabs.SlabGeometry(sc.para, sc.grid_space, sc.ext(), 2)
    assert g.halo == 8 and g.edges == [0, 30, 60]
    own = g.owner(torch.from_numpy(sc.pos)).numpy()
    assert set(own.tolist()) == {0, 1}
    # the column of a particle is the solver's: float32 (x - gmin) * (1 / cell), truncated
    ix = ((sc.pos[:, 0] - np.float32(sc.grid_space[0])) * g.inv_cell).astype(np.int32)
    assert np.array_equal(own, (ix >= 30).astype(np.int32))
    with pytest.raises(ValueError):
        slabs.SlabGeometry(sc.para, sc.grid_space, sc.ext(), 8)  # slabs narrower than the halo
    out = sc.pos.copy()
    out[0, 1] = -1.0
    with pytest.raises(ValueError):
        g.owner(torch.from_numpy(out))


def test_pack_round_trip():
    rng = np.random.RandomState(0)
    p = slabs.Part(torch.from_numpy(rng.randn(5, 3).astype(np.float32)),
                   torch.from_numpy(rng.randn(5, 3).astype(np.float32)),
                   torch.arange(5, dtype=torch.int32), torch.arange(5, dtype=torch.int32) * 7,
                   torch.arange(5, dtype=torch.int32) % 2)
    q = slabs.Part.unpack(p.pack())
    for f in ("pos", "vel", "gid", "key", "rank"):
        assert torch.equal(getattr(p, f), getattr(q, f))


def test_two_ranks_match_single_domain_bitexact():
    steps = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pos, vel = next((a, b) for a, b, _ in got if a is not None)
    counts = [c for _, _, c in got]
    sc = slab_scene()
    assert sum(c[-1] for c in counts) == sc.n and min(c[-1] for c in counts) > 0
    assert counts[1][-1] != counts[1][0]  # particles crossed the face
    o = O.Oracle(O.params_for_scene(sc), sc.pos, sc.vel)
    o.substep(steps)
    perm = o.get("perm")
    want_x = np.empty((sc.n, 3), np.float32)
    want_v = np.empty((sc.n, 3), np.float32)
    want_x[perm] = o.get("x").astype(np.float32)
    want_v[perm] = o.get("v").astype(np.float32)
    assert np.array_equal(pos.view(np.uint32), want_x.view(np.uint32))
    assert np.array_equal(vel.view(np.uint32), want_v.view(np.uint32))


def test_fast_particle_beyond_the_ghost_zone_is_an_error():
    """A particle that moves farther along x in one substep than the halo's
    margin (halo - reach) could leave a neighbourhood incomplete; the slab step
    raises instead of returning a state that differs from the single domain."""
    sc = slab_scene(iterations=2)
    g = slabs.SlabGeometry(sc.para, sc.grid_space, sc.ext(), 2)
    assert g.reach == 6 and g.margin == 2
    vel = sc.vel.copy()
    vel[0, 0] = 100.0  # 100 * dt = 0.83 = 8 cell columns in one substep
    group = slabs.SlabGroup(g, [OracleEngine(sc), OracleEngine(sc)])
    group.load(torch.from_numpy(sc.pos), torch.from_numpy(vel))
    with pytest.raises(RuntimeError, match="cell columns"):
        group.step(1)
    with pytest.raises(ValueError):
        slabs.SlabGeometry(sc.para, sc.grid_space, sc.ext(), 2, halo_h=6)  # no margin beyond the reach
