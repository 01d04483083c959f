"""The library behind the reference's own entry points, called as the reference
app calls them (GPU test).

oracle/_ref/ref_app_driver is a C++ program compiled against the reference's
headers (kernels/cudaPBF.h, include/solverBase.h, include/AABB.h) and linked
with pbf_b200/csrc/reference_shim.cpp and libpbf_b200.so. It does what
src/renderapp.cpp:246-251 and :499 do: the caller cudaMallocs data.position,
calls initCUDASolverDataBuffer once and cudaPBFSolve(data, para) once per frame,
and reads data.position after each call. Every frame must equal the oracle bit
for bit (the shim's defaults are the reference's constants: gravity -49, a 64^3
grid, 63 neighbours, the reference formulas), including frames after `para`
changes between calls, which the reference honours on every call
(kernels/cudaPBF.cu:50-115).
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import scenes

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(REPO, "oracle", "_ref", "ref_app_driver")


def para_bytes(p) -> bytes:
    return bytes(memoryview(p))


def run_driver(tmp_path, sc, calls, change_at, para2):
    inp = tmp_path / "in.bin"
    out = tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<iii", sc.n, calls, change_at))
        f.write(para_bytes(sc.para))
        f.write(para_bytes(para2))
        f.write(np.asarray(sc.grid_space, np.float32).tobytes())
        f.write(np.asarray(sc.boundary, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.pos, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.vel, np.float32).tobytes())
    r = subprocess.run([DRIVER, str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    frames = np.fromfile(out, np.float32).reshape(calls + 1, sc.n, 3)
    return frames, r.stderr


def oracle_frames(sc, calls, change_at, para2):
    orc = O.Oracle(O.params_from(sc.para, sc.grid_space, sc.boundary), sc.pos, sc.vel)
    frames = [sc.pos.astype(np.float32)]
    for k in range(1, calls + 1):
        if k == change_at:
            orc.set_params(O.params_from(para2, sc.grid_space, sc.boundary))
        orc.substep()
        x = orc.get("x")
        perm = orc.get("perm")
        out = np.empty_like(x)
        out[perm] = x
        frames.append(out.astype(np.float32))
    return frames


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="reference app driver not built (needs the reference headers)")
@pytest.mark.parametrize("block", [16, 32])
def test_reference_entry_points_as_the_app_calls_them(tmp_path, block):
    sc = scenes.dam_break(block, (40, 20, 20), stable=False, gravity=-49.0, iterations=4)
    para2 = scenes.benchmark_parameter(sc.n, iterations=2)
    para2.dt = np.float32(0.006)
    para2.invDt = np.float32(1.0) / para2.dt
    calls, change_at = 4, 3
    got, err = run_driver(tmp_path, sc, calls, change_at, para2)
    assert "pbf_b200:" not in err, err
    want = oracle_frames(sc, calls, change_at, para2)
    for k in range(calls + 1):
        bad = got[k].view(np.uint32) != want[k].view(np.uint32)
        assert not bad.any(), f"frame {k}: {int(bad.sum())} values differ"
    # the parameter change took effect: the frames after it differ from a run without it
    same, _ = run_driver(tmp_path, sc, calls, calls + 1, para2)
    assert np.array_equal(same[:change_at].view(np.uint32), got[:change_at].view(np.uint32))
    assert not np.array_equal(same[change_at].view(np.uint32), got[change_at].view(np.uint32))


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="reference app driver not built (needs the reference headers)")
def test_reference_entry_points_report_failures(tmp_path):
    """A parameter the library rejects is printed to stderr by the shim, and the
    frames keep the last good state instead of changing silently."""
    sc = scenes.dam_break(12, (40, 20, 20), stable=False, gravity=-49.0, iterations=2)
    bad = scenes.benchmark_parameter(sc.n, iterations=2)
    bad.iterations = 99  # beyond the library's 64
    got, err = run_driver(tmp_path, sc, 2, 2, bad)
    assert "pbf_set_parameter failed" in err
    assert np.array_equal(got[1].view(np.uint32), got[2].view(np.uint32))
