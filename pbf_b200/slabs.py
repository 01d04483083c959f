"""One scene split over x-slabs of cells, one slab per rank (no reference
counterpart: the reference solves one scene on one device).

Slab r owns the particles whose cell lies in columns [edges[r], edges[r+1]) of
the global grid; the grid must cover the walls, so that no particle is ever
outside it. Each substep a rank gathers, besides its own particles, the
particles of its neighbours that lie within `halo` cells of its faces, runs the
unchanged CUDA substep on that set and keeps the particles that end the
substep in its slab. This is a ghost zone wide enough that no exchange is
needed inside the substep: a particle's result depends only on particles
within (2 iterations + 2) h of it (lambda and the correction each reach h per
Jacobi iteration, then curl and vorticity), so with the default halo of
(2 iterations + 4) h every particle a rank keeps is computed from a complete
neighbourhood. One exchange per substep (the faces' particles to the two
neighbours) is the whole communication.

The results are those of the single-domain solver bit for bit. The local grid
is the global grid (same origin, cell size and keys), so the cells, the 63-entry
cap and the neighbour lists (slots in ascending order) are the same; and the
local set is uploaded in the global slot order, which the substep's stable
sort needs: particles are merged by (key, rank) of the cell they were sorted
into last substep, a unique and totally ordered label (a cell and its halo
copy are sorted identically on every rank that holds it).

`SlabRank` is one rank's state and step; `SlabGroup` runs all slabs of a scene
in one process (on one device, exchanging by tensor copies), and `DistComm`
carries the exchange over torch.distributed point-to-point (NCCL between GPUs,
gloo on CPU).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np


@dataclass
class Part:
    """Particles in slot order: pos, vel (m x 3 float32), gid (global index),
    key and rank (int32: the cell they were sorted into last substep and their
    slot within it)."""
    pos: "object"
    vel: "object"
    gid: "object"
    key: "object"
    rank: "object"

    def __len__(self) -> int:
        return int(self.gid.shape[0])

    def take(self, idx) -> "Part":
        return Part(self.pos[idx], self.vel[idx], self.gid[idx], self.key[idx], self.rank[idx])

    @staticmethod
    def cat(parts: Sequence["Part"]) -> "Part":
        import torch
        return Part(*(torch.cat([getattr(p, f) for p in parts]) for f in ("pos", "vel", "gid", "key", "rank")))

    def pack(self):
        """One int32 tensor m x 9 (the floats as their bits)."""
        import torch
        f = torch.cat([self.pos, self.vel], dim=1).contiguous().view(torch.int32)
        return torch.cat([f, self.gid[:, None], self.key[:, None], self.rank[:, None]], dim=1).contiguous()

    @staticmethod
    def unpack(t) -> "Part":
        import torch
        f = t[:, :6].contiguous().view(torch.float32)
        return Part(f[:, :3].contiguous(), f[:, 3:].contiguous(), t[:, 6].contiguous(), t[:, 7].contiguous(),
                    t[:, 8].contiguous())


class SlabGeometry:
    """Cell columns of each slab and the cell arithmetic of the solver."""

    def __init__(self, para, grid_space: Sequence[float], ext, nslabs: int, halo_h: Optional[float] = None):
        f32 = np.float32
        self.dims = [int(d) for d in ext.grid_dims]
        cs = f32(f32(para.h) * f32(ext.cell_scale))
        self.inv_cell = f32(1.0) / cs  # as the solver computes it (pbf_capi.cu: make_kparams)
        self.gmin = np.asarray(grid_space[:3], f32)
        if halo_h is None:
            halo_h = 2 * int(para.iterations) + 4
        self.halo = int(math.ceil(halo_h / float(ext.cell_scale) - 1e-9))
        # cell columns a result depends on (lambda and the correction reach h per
        # Jacobi iteration, curl and vorticity h each), and what the halo leaves
        # beyond that for motion within a substep
        self.reach = int(math.ceil((2 * int(para.iterations) + 2) / float(ext.cell_scale) - 1e-9))
        self.margin = self.halo - self.reach
        if self.margin < 1:
            raise ValueError(f"a halo of {self.halo} cell columns leaves no margin beyond the reach of "
                             f"{self.reach} columns")
        nx = self.dims[0]
        self.edges = [round(r * nx / nslabs) for r in range(nslabs + 1)]
        self.nslabs = nslabs
        widths = [self.edges[r + 1] - self.edges[r] for r in range(nslabs)]
        if nslabs > 1 and min(widths) < self.halo:
            raise ValueError(f"slabs of {min(widths)} cell columns are narrower than the halo ({self.halo})")

    def cells(self, pos):
        """Cell column index and whether the particle is inside the grid (the
        solver's cell_dims / cell_key: float32 (x - gmin) * inv_cell, truncated)."""
        import torch
        g = torch.as_tensor(self.gmin, device=pos.device)
        d = ((pos - g) * float(self.inv_cell)).to(torch.int32)
        dims = torch.as_tensor(self.dims, device=pos.device, dtype=torch.int32)
        inside = ((d >= 0) & (d < dims)).all(dim=1)
        return d[:, 0], inside

    def owner(self, pos):
        """Slab of each particle; raises when one is outside the grid."""
        import torch
        ix, inside = self.cells(pos)
        if not bool(inside.all()):
            raise ValueError("slab decomposition needs every particle inside the grid (a grid covering the walls)")
        e = torch.as_tensor(self.edges[1:-1], device=pos.device, dtype=torch.int32)
        return torch.bucketize(ix.contiguous(), e, right=True).to(torch.int32)


class SlabRank:
    """The particles of slab r and one substep of them."""

    def __init__(self, geom: SlabGeometry, r: int, engine):
        self.geom, self.r, self.engine = geom, r, engine
        self.own: Optional[Part] = None

    def load(self, pos, vel):
        """This slab's particles of the global arrays (same on every rank), in
        global order (the order of an upload)."""
        import torch
        gid = torch.arange(pos.shape[0], device=pos.device, dtype=torch.int32)
        keep = self.geom.owner(pos) == self.r
        self.own = Part(pos[keep].contiguous(), vel[keep].contiguous(), gid[keep], torch.zeros_like(gid[keep]),
                        gid[keep])

    def sends(self):
        """The particles within the halo of the left and of the right face."""
        g, r = self.geom, self.r
        ix, _ = g.cells(self.own.pos)
        take = lambda m: self.own.take(m.nonzero().squeeze(1))  # noqa: E731
        left = take(ix < g.edges[r] + g.halo) if r > 0 else None
        right = take(ix >= g.edges[r + 1] - g.halo) if r < g.nslabs - 1 else None
        return left, right

    def step(self, from_left: Optional[Part], from_right: Optional[Part]):
        """One substep of the own particles with the neighbours' face particles."""
        import torch
        parts = [p for p in (from_left, self.own, from_right) if p is not None and len(p) > 0]
        if not parts:
            return
        local = Part.cat(parts)
        order = torch.sort((local.key.to(torch.int64) << 32) | local.rank.to(torch.int64), stable=True).indices
        local = local.take(order)
        pos, vel, ids, key, rank = self.engine.run(local.pos.contiguous(), local.vel.contiguous())
        res = Part(pos, vel, local.gid[ids.long()], key, rank)
        keep = (self.geom.owner(pos) == self.r).nonzero().squeeze(1)
        self.check_ghost_zone(local.pos[ids.long()], pos, keep)
        self.own = res.take(keep)

    def check_ghost_zone(self, start, end, keep):
        """The ghost zone is exact only while no particle moves farther than the
        halo's margin (halo - reach cell columns) along x in one substep: a faster
        one could start outside every halo and end in a neighbourhood, or a kept
        particle could have started too deep in the halo for its neighbourhood to
        be complete. Every rank checks the particles it computed (each particle
        is owned, so computed completely, by some rank), and raises instead of
        returning a state that would differ from the single-domain solver."""
        g, r = self.geom, self.r
        x0, _ = g.cells(start)
        x1, _ = g.cells(end)
        moved = int((x1 - x0).abs().max().item()) if x0.numel() else 0
        if moved > g.margin:
            raise RuntimeError(f"slab {r}: a particle moved {moved} cell columns in one substep, more than the "
                               f"ghost zone's margin of {g.margin}; use a wider halo (halo_h) or a smaller dt")
        if keep.numel():
            k0 = x0[keep]
            lo, hi = g.edges[r] - g.margin, g.edges[r + 1] + g.margin
            if bool(((k0 < lo) | (k0 >= hi)).any()):
                raise RuntimeError(f"slab {r}: a particle it keeps started deeper in the halo than the margin of "
                                   f"{g.margin} cell columns, so its neighbourhood was incomplete")


class SlabGroup:
    """All slabs of one scene in one process (an emulation of the ranks on one
    device: the exchange is a tensor copy)."""

    def __init__(self, geom: SlabGeometry, engines: List):
        self.geom = geom
        self.ranks = [SlabRank(geom, r, e) for r, e in enumerate(engines)]

    def load(self, pos, vel):
        for s in self.ranks:
            s.load(pos, vel)

    def step(self, substeps: int = 1):
        for _ in range(substeps):
            sends = [s.sends() for s in self.ranks]
            for r, s in enumerate(self.ranks):
                left = sends[r - 1][1] if r > 0 else None
                right = sends[r + 1][0] if r < len(self.ranks) - 1 else None
                s.step(left, right)

    def gather(self):
        """Global positions and velocities by particle index."""
        return gather_parts([s.own for s in self.ranks])


def gather_parts(parts: Sequence[Part]):
    import torch
    allp = Part.cat([p for p in parts if p is not None and len(p) > 0])
    order = torch.argsort(allp.gid.long())
    return allp.pos[order], allp.vel[order]


class DistComm:
    """The per-substep exchange of a slab over torch.distributed (the process
    group's backend: NCCL for device tensors, gloo for CPU tensors)."""

    def __init__(self, rank: int, world: int, device):
        self.rank, self.world, self.device = rank, world, device

    def _swap(self, to_left: Optional[Part], to_right: Optional[Part]):
        import torch
        import torch.distributed as dist
        r, w = self.rank, self.world
        empty = torch.empty((0, 9), dtype=torch.int32, device=self.device)
        out = {"l": to_left.pack() if to_left is not None else empty,
               "r": to_right.pack() if to_right is not None else empty}
        # sizes first, then the payloads (every rank takes the same steps)
        n_send = {k: torch.tensor([v.shape[0]], dtype=torch.int64, device=self.device) for k, v in out.items()}
        n_recv = {k: torch.zeros(1, dtype=torch.int64, device=self.device) for k in ("l", "r")}
        ops = []
        if r > 0:
            ops += [dist.P2POp(dist.isend, n_send["l"], r - 1), dist.P2POp(dist.irecv, n_recv["l"], r - 1)]
        if r < w - 1:
            ops += [dist.P2POp(dist.isend, n_send["r"], r + 1), dist.P2POp(dist.irecv, n_recv["r"], r + 1)]
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        got = {k: torch.empty((int(n_recv[k].item()), 9), dtype=torch.int32, device=self.device) for k in ("l", "r")}
        ops = []
        if r > 0:
            if out["l"].shape[0]:
                ops.append(dist.P2POp(dist.isend, out["l"], r - 1))
            if got["l"].shape[0]:
                ops.append(dist.P2POp(dist.irecv, got["l"], r - 1))
        if r < w - 1:
            if out["r"].shape[0]:
                ops.append(dist.P2POp(dist.isend, out["r"], r + 1))
            if got["r"].shape[0]:
                ops.append(dist.P2POp(dist.irecv, got["r"], r + 1))
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        return (Part.unpack(got["l"]) if r > 0 else None), (Part.unpack(got["r"]) if r < w - 1 else None)

    def step(self, slab: SlabRank, substeps: int = 1):
        for _ in range(substeps):
            to_left, to_right = slab.sends()
            from_left, from_right = self._swap(to_left, to_right)
            slab.step(from_left, from_right)

    def gather(self, slab: SlabRank):
        """Global positions and velocities by particle index, on every rank."""
        import torch
        import torch.distributed as dist
        t = slab.own.pack()
        n = torch.tensor([t.shape[0]], dtype=torch.int64, device=self.device)
        sizes = [torch.zeros_like(n) for _ in range(self.world)]
        dist.all_gather(sizes, n)
        m = max(int(s.item()) for s in sizes)
        pad = torch.zeros((m, 9), dtype=torch.int32, device=self.device)
        pad[: t.shape[0]] = t
        allt = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(allt, pad)
        parts = [Part.unpack(a[: int(s.item())]) for a, s in zip(allt, sizes)]
        return gather_parts(parts)


class CudaEngine:
    """The CUDA substep of a slab's particle set (a single-scene solver created
    for `capacity` particles and resized to each set)."""

    def __init__(self, para, grid_space, boundary, ext, capacity: int):
        import copy

        from .solver import Solver
        if ext.adaptive or ext.warm_start:
            raise ValueError("slabs run plain Jacobi iterations (no adaptive loop, no warm start)")
        p = copy.copy(para)
        p.nParticles = int(capacity)
        self.solver = Solver(p, grid_space, boundary, ext)

    def run(self, pos, vel):
        """One substep of (pos, vel) (device tensors, m x 3, in upload order);
        returns the state in slot order: pos, vel, ids (upload index), key, rank."""
        import torch
        m = int(pos.shape[0])
        s = self.solver
        s.resize(m)
        s.upload_device(pos, vel)
        s.step(1)
        out = (torch.empty_like(pos), torch.empty_like(vel),
               *(torch.empty(m, dtype=torch.int32, device=pos.device) for _ in range(3)))
        s.download_sorted_device(*out)
        return out
