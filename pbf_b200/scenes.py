"""Seeded synthetic scenes (jittered particle lattices) and their parameters.

* dam_break(): the single-block dam break of the benchmark workloads (a cubic
  lattice at spacing 0.5h in a box corner, uniform jitter of +-0.01h drawn from
  MT19937).
* reference_app_scene(): the five initial conditions of the reference app
  (src/renderapp.cpp:115-234) with a seeded generator in place of rand().
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._lib import PBF_FLAG_CLAMP_C, PBF_FLAG_WALL_DENSITY, PBF_FLAG_XSPH_RHO, ExtParams, SolverParameter
from .solver import default_ext, make_parameter


@dataclass
class Scene:
    name: str
    para: SolverParameter
    grid_space: list
    boundary: list
    ext_overrides: dict
    pos: np.ndarray
    vel: np.ndarray
    info: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def ext(self, **more) -> ExtParams:
        kw = dict(self.ext_overrides)
        kw.update(more)
        return default_ext(**kw)


def benchmark_parameter(n: int, h: float = 0.1, iterations: int = 4, substeps_per_frame: int = 2) -> SolverParameter:
    """h=0.1, rho0=6378, eps=600, s_corr k=0.1 n=4 dq=0.2h, XSPH c=0.01,
    vorticity eps=0.0005, dt = (1/60) / substeps_per_frame."""
    dt = np.float32(1.0 / 60.0) / np.float32(substeps_per_frame)
    return make_parameter(h=h, nParticles=n, restRho=6378.0, epsilon=600.0, k=0.1, n=4.0,
                          deltaq=np.float32(0.2) * np.float32(h), c=0.01, dt=float(dt), iterations=iterations,
                          vorticityConfinementEpilon=0.0005, radius=np.float32(0.3) * np.float32(h))


def lattice_block(counts, spacing: float, origin, rng: np.random.RandomState, jitter: float) -> np.ndarray:
    """x-fastest lattice (the reference app's index order, src/renderapp.cpp:143-151)."""
    nx, ny, nz = counts
    i = np.arange(nx * ny * nz)
    idx = np.stack([i % nx, (i // nx) % ny, i // (nx * ny)], axis=1).astype(np.float64)
    pos = np.asarray(origin, np.float64) + spacing * idx
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos.astype(np.float32)


def stable_overrides(para: SolverParameter) -> dict:
    """Named departures for long runs (the reference formulas diverge at these
    parameters within a few substeps): unilateral density constraint, XSPH
    weighted by 1/rho0, walls that carry the density of a fluid half-space, and
    s_corr expressed in lambda units, i.e. divided by (sum |grad C|^2 + eps) of a
    rest lattice at spacing 0.5h."""
    g = rest_gradient_sum(float(para.h), float(para.restRho), 0.5 * float(para.h))
    return {"flags": PBF_FLAG_CLAMP_C | PBF_FLAG_XSPH_RHO | PBF_FLAG_WALL_DENSITY,
            "scorr_scale": float(1.0 / (g + float(para.epsilon)))}


def rest_gradient_sum(h: float, rho0: float, spacing: float) -> float:
    """sum_j |grad W_spiky(r_j)|^2 / rho0^2 + |sum_j grad W|^2 / rho0^2 over a
    simple cubic lattice at `spacing` (the second term is zero by symmetry)."""
    r = int(np.ceil(h / spacing))
    g = np.arange(-r, r + 1) * spacing
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    d = np.sqrt(X**2 + Y**2 + Z**2).ravel()
    d = d[(d > 0) & (d <= h)]
    c = 45.0 / (np.pi * h**6)
    mag = c * (h - d) ** 2
    return float(np.sum(mag**2) / rho0**2)


def dam_break(block: int = 32, box_cells=(40, 20, 20), h: float = 0.1, seed: int = 0, gravity: float = -9.8,
              iterations: int = 4, stable: bool = True, grid_dims: Optional[tuple] = None,
              jitter: float = 0.01) -> Scene:
    """block^3 lattice at spacing 0.5h, origin one spacing from the box corner,
    jitter U(+-0.01h); box = box_cells * h with its minimum corner at the origin."""
    spacing = 0.5 * h
    rng = np.random.RandomState(seed)
    pos = lattice_block((block, block, block), spacing, (spacing, spacing, spacing), rng, jitter * h)
    n = pos.shape[0]
    vel = np.zeros_like(pos)
    para = benchmark_parameter(n, h=h, iterations=iterations)
    box = [0.0, 0.0, 0.0, box_cells[0] * h, box_cells[1] * h, box_cells[2] * h]
    r = float(para.radius)
    bd = [box[0] + r, box[1] + r, box[2] + r, box[3] - r, box[4] - r, box[5] - r]
    dims = list(grid_dims) if grid_dims is not None else list(box_cells)
    ov = {"gravity": (0.0, gravity, 0.0), "grid_dims": dims}
    if stable:
        ov.update(stable_overrides(para))
    return Scene(f"dam_break_{block}^3", para, box, bd, ov, pos, vel,
                 info={"block": block, "box_cells": list(box_cells), "seed": seed, "stable": stable})


def config0(seed: int = 0, stable: bool = True, **kw) -> Scene:
    """32,768 particles: 32^3 block in a 40h x 20h x 20h box."""
    return dam_break(32, (40, 20, 20), seed=seed, stable=stable, **kw)


def config1(seed: int = 0, stable: bool = True, **kw) -> Scene:
    """262,144 particles: 64^3 block in an 80h x 40h x 40h box."""
    return dam_break(64, (80, 40, 40), seed=seed, stable=stable, **kw)


def reference_app_scene(idx: int, seed: int = 0, dims=(64, 64, 64)) -> Scene:
    """Scenes 1-5 of src/renderapp.cpp:137-234 (h=1, rho0=6, eps=1, k=0.01,
    dq=0.1h, n=4, c=0.1, dt=0.016, 4 iterations, vorticity eps 0.1, radius 0.3;
    box [-30,30]x[0,40]x[-30,30]). The per-particle jitter 0.2*rand()/RAND_MAX is
    drawn from a seeded generator."""
    nx, ny, nz = dims
    n = nx * ny * nz
    para = make_parameter(h=1.0, nParticles=n, restRho=6.0, epsilon=1.0, k=0.01, deltaq=0.1, n=4.0, c=0.1,
                          dt=0.016, iterations=4, vorticityConfinementEpilon=0.1, radius=0.3)
    box = [-30.0, 0.0, -30.0, 30.0, 40.0, 30.0]
    r = 0.3
    bd = [box[0] + r, box[1] + r, box[2] + r, box[3] - r, box[4] - r, box[5] - r]
    rng = np.random.RandomState(seed)

    def region(lo, hi, count, cnt_y=None):
        gap = (np.asarray(hi, np.float32) - np.asarray(lo, np.float32)) / np.asarray(dims, np.float32)
        i = np.arange(count)
        cy = ny if cnt_y is None else cnt_y
        d = np.stack([i % nx, (i // nx) % cy, i // (nx * cy)], axis=1).astype(np.float32)
        p = np.asarray(lo, np.float32) + d * gap
        return (p + np.float32(0.2) * rng.uniform(0, 1, size=p.shape).astype(np.float32)).astype(np.float32)

    if idx == 1:
        pos = region((-16.0, 0.2, -16.0), (16.0, 32.2, 16.0), n)
        vel = np.tile(np.float32([0.0, 20.0, 0.0]), (n, 1))
    elif idx == 2:
        pos = region((-28.0, 0.3, -4.0), (4.0, 32.3, 28.0), n)
        vel = np.tile(np.float32([0.0, 0.0, -20.0]), (n, 1))
    elif idx == 3:
        half = n // 2
        a = region((-29.7, 0.2, -29.7), (-2.0, 32.2, -2.0), half, cnt_y=32)
        # the second block reuses the first block's spacing (src/renderapp.cpp:190-203)
        gap = (np.float32([-2.0, 32.2, -2.0]) - np.float32([-29.7, 0.2, -29.7])) / np.asarray(dims, np.float32)
        i = np.arange(half)
        d = np.stack([i % nx, (i // nx) % 32, i // (nx * 32)], axis=1).astype(np.float32)
        b = np.float32([2.0, 0.2, 2.0]) + d * gap
        b = (b + np.float32(0.2) * rng.uniform(0, 1, size=b.shape).astype(np.float32)).astype(np.float32)
        pos = np.concatenate([a, b])
        vel = np.concatenate([np.tile(np.float32([50.0, 0.0, 50.0]), (half, 1)),
                              np.tile(np.float32([-50.0, 0.0, -50.0]), (half, 1))])
    elif idx == 4:
        pos = region((-24.0, 0.2, -16.0), (8.0, 32.2, 16.0), n)
        vel = np.tile(np.float32([-10.0, 15.0, 0.0]), (n, 1))
    elif idx == 5:
        pos = region((-16.0, 0.2, -16.0), (16.0, 32.2, 16.0), n)
        # 50 * normalize(-(-z, 0, x)), src/renderapp.cpp:229
        t = -np.stack([-pos[:, 2], np.zeros(n, np.float32), pos[:, 0]], axis=1)
        nrm = np.linalg.norm(t, axis=1, keepdims=True)
        vel = (50.0 * t / np.maximum(nrm, 1e-30)).astype(np.float32)
    else:
        raise ValueError("scene index must be 1..5")
    ov = {"gravity": (0.0, -49.0, 0.0), "grid_dims": [64, 64, 64]}
    return Scene(f"reference_app_scene_{idx}", para, box, bd, ov, pos.astype(np.float32), vel.astype(np.float32),
                 info={"scene": idx, "seed": seed})


# ---- batches of independent scenes --------------------------------------------
def random_block_scene(n: int, rng: np.random.RandomState, h: float = 0.1, iterations: int = 4,
                       stable: bool = True, jitter: float = 0.01) -> Scene:
    """n particles in a cube-ish jittered lattice block (x-fastest, spacing 0.5h)
    at a random position on the floor of a box twice the block's size, stretched
    in x by an aspect ratio drawn from U[1, 3]."""
    spacing = 0.5 * h
    m = max(2, int(round(n ** (1.0 / 3.0))))
    counts = (m, m, int(np.ceil(n / (m * m))))
    extent = [c * spacing for c in counts]
    side = 2.0 * max(extent) + 4 * spacing
    aspect = rng.uniform(1.0, 3.0)
    cells = (int(np.ceil(side * aspect / h)), int(np.ceil(side / h)), int(np.ceil(side / h)))
    box = [0.0, 0.0, 0.0, cells[0] * h, cells[1] * h, cells[2] * h]
    origin = (rng.uniform(spacing, box[3] - extent[0] - spacing), spacing + rng.uniform(0.0, 0.25 * box[4]),
              rng.uniform(spacing, box[5] - extent[2] - spacing))
    pos = lattice_block(counts, spacing, origin, rng, jitter * h)[:n]
    vel = np.zeros_like(pos)
    para = benchmark_parameter(n, h=h, iterations=iterations)
    r = float(para.radius)
    bd = [box[0] + r, box[1] + r, box[2] + r, box[3] - r, box[4] - r, box[5] - r]
    ov = {"gravity": (0.0, -9.8, 0.0), "grid_dims": list(cells)}
    if stable:
        ov.update(stable_overrides(para))
    return Scene(f"block_{n}", para, box, bd, ov, pos, vel, info={"aspect": aspect, "counts": counts})


def config2(seed: int = 0, n_scenes: int = 64, lo: int = 4096, hi: int = 65536, iterations: int = 4,
            stable: bool = True) -> list:
    """64 scenes with particle counts log-uniform in [4,096, 65,536] (seeded)."""
    rng = np.random.RandomState(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_scenes)).round().astype(int)
    return [random_block_scene(int(c), rng, iterations=iterations, stable=stable) for c in counts]


def config4(seed: int = 0, block: int = 128, iterations: int = 4, stable: bool = True, small: int = 65536,
            n_small: int = 8) -> list:
    """Double dam break: two block^3 jittered lattices facing each other in a
    320h x 160h x 160h box with a static sphere of radius 20h at the centre,
    batched with n_small scenes of `small` particles."""
    h = 0.1
    spacing = 0.5 * h
    rng = np.random.RandomState(seed)
    cells = (320, 160, 160)
    box = [0.0, 0.0, 0.0, cells[0] * h, cells[1] * h, cells[2] * h]
    ext = block * spacing
    zc = 0.5 * (box[5] - ext)
    a = lattice_block((block, block, block), spacing, (spacing, spacing, zc), rng, 0.01 * h)
    b = lattice_block((block, block, block), spacing, (box[3] - ext, spacing, zc), rng, 0.01 * h)
    pos = np.concatenate([a, b])
    n = pos.shape[0]
    para = benchmark_parameter(n, h=h, iterations=iterations)
    r = float(para.radius)
    bd = [box[0] + r, box[1] + r, box[2] + r, box[3] - r, box[4] - r, box[5] - r]
    sphere = (0.5 * box[3], 20 * h, 0.5 * box[5], 20 * h)
    ov = {"gravity": (0.0, -9.8, 0.0), "grid_dims": list(cells), "sphere": sphere}
    if stable:
        ov.update(stable_overrides(para))
    big = Scene(f"double_dam_break_{n}", para, box, bd, ov, pos, np.zeros_like(pos), info={"sphere": sphere})
    return [big] + [random_block_scene(small, rng, iterations=iterations, stable=stable) for _ in range(n_small)]


def batch_inputs(scenes: list, iterations: Optional[int] = None):
    """(SolverParameter, scene descriptions, ext overrides, positions, velocities)
    for a BatchSolver over `scenes`; they share parameters and flags."""
    total = sum(s.n for s in scenes)
    p0 = scenes[0].para
    para = benchmark_parameter(total, h=float(p0.h), iterations=int(p0.iterations if iterations is None else iterations))
    descs = []
    for s in scenes:
        descs.append({"grid_space": s.grid_space, "boundary": s.boundary, "grid_dims": s.ext_overrides["grid_dims"],
                      "nparticles": s.n, "sphere": s.ext_overrides.get("sphere", (0.0, 0.0, 0.0, 0.0))})
    ov = {k: v for k, v in scenes[0].ext_overrides.items() if k not in ("grid_dims", "sphere")}
    pos = np.concatenate([s.pos for s in scenes])
    vel = np.concatenate([s.vel for s in scenes])
    return para, descs, ov, pos, vel
