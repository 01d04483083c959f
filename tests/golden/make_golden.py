"""Generates the golden fixtures of the reference's own solvers.

  python tests/golden/make_golden.py cpu [outdir]   reference CPU solver (oracle/_ref/libpbfref_cpu.so)
  python tests/golden/make_golden.py gpu [outdir]   reference CUDA solver (oracle/_ref/libpbfref_gpu.so, needs a GPU)

Both run the unmodified reference code on the seeded 16^3 dam-break lattice
(4,096 particles, h = 0.1, box 40h x 20h x 20h, reference 64^3 grid) and store
its outputs as compressed .npz next to this script (or in outdir).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from pbf_b200 import scenes  # noqa: E402


def make_cpu(outdir):
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    sc.para.iterations = 4
    ref = O.RefCpu(sc.para, sc.grid_space)
    p, v = ref.solve(sc.pos, sc.vel, substeps=2)
    out = dict(pos_in=sc.pos, iterations=np.int32(4), substeps=np.int32(2), x=p, v=v)
    for name in ("lambda", "dp", "curl", "vort", "visc"):
        out[name] = ref.get(name).astype(np.float32)
    for name in ("start", "end", "ncnt"):
        out[name] = ref.get(name)
    np.savez_compressed(os.path.join(outdir, "refcpu_dam16.npz"), **out)


def make_gpu(outdir):
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    for iters in (1, 4):
        sc.para.iterations = iters
        r = O.refgpu_run(sc.para, sc.grid_space, sc.boundary, sc.pos, sc.vel, substeps=1)
        grid = r.pop("grid")
        nz = np.nonzero(grid[:, 1] > grid[:, 0])[0].astype(np.int32)
        r["grid_cells"] = nz
        r["grid_start"] = grid[nz, 0].astype(np.int32)
        r["grid_end"] = grid[nz, 1].astype(np.int32)
        r.pop("prefix")
        r["pos_in"] = sc.pos
        r["iterations"] = np.int32(iters)
        np.savez_compressed(os.path.join(outdir, f"refgpu_dam16_it{iters}.npz"), **r)


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "cpu"
    outdir = sys.argv[2] if len(sys.argv) > 2 else HERE
    os.makedirs(outdir, exist_ok=True)
    (make_cpu if which == "cpu" else make_gpu)(outdir)
