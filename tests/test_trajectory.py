"""Trajectory files (pbf_b200.trajectory): round trip, header, partial files
(CPU tests), and a recorded GPU run that a second run reproduces frame for frame."""
import os

import numpy as np
import pytest

from pbf_b200 import scenes
from pbf_b200.trajectory import HEADER_BYTES, TrajectoryReader, TrajectoryWriter, record


def _scene():
    return scenes.dam_break(6, (40, 20, 20), stable=True, iterations=2)


def test_round_trip(tmp_path):
    sc = _scene()
    rng = np.random.RandomState(0)
    frames = [(3 * k, rng.randn(sc.n, 3).astype(np.float32), rng.randn(sc.n, 3).astype(np.float32)) for k in range(5)]
    path = os.path.join(tmp_path, "t.pbft")
    with TrajectoryWriter(path, sc.para, sc.grid_space, sc.boundary, sc.n) as w:
        for s, p, v in frames:
            w.write(s, p, v)
    r = TrajectoryReader(path)
    assert len(r) == 5 and r.n == sc.n
    assert bytes(r.para) == bytes(sc.para)
    assert np.array_equal(r.grid_space, np.float32(sc.grid_space)) and np.array_equal(r.boundary, np.float32(sc.boundary))
    for (s, p, v), (s2, p2, v2) in zip(frames, r):
        assert s == s2 and np.array_equal(p, p2) and np.array_equal(v, v2)
    assert r[-1][0] == 12


def test_positions_only_and_unclosed_file(tmp_path):
    sc = _scene()
    path = os.path.join(tmp_path, "p.pbft")
    w = TrajectoryWriter(path, sc.para, sc.grid_space, sc.boundary, sc.n, velocities=False)
    for k in range(3):
        w.write(k, sc.pos + k)
    w._f.flush()  # a run that stopped before close(): the header still says 0 frames
    r = TrajectoryReader(path)
    assert len(r) == 3 and r[2][2] is None and np.array_equal(r[2][1], sc.pos + 2)
    w.close()
    assert len(TrajectoryReader(path)) == 3
    # a torn last frame is not reported
    with open(path, "ab") as f:
        f.write(b"\0" * 20)
    assert len(TrajectoryReader(path)) == 3


def test_rejects_bad_files_and_shapes(tmp_path):
    sc = _scene()
    bad = os.path.join(tmp_path, "bad.pbft")
    with open(bad, "wb") as f:
        f.write(b"x" * HEADER_BYTES)
    with pytest.raises(ValueError):
        TrajectoryReader(bad)
    with TrajectoryWriter(os.path.join(tmp_path, "s.pbft"), sc.para, sc.grid_space, sc.boundary, sc.n) as w:
        with pytest.raises(ValueError):
            w.write(0, sc.pos[:-1], sc.vel[:-1])
        with pytest.raises(ValueError):
            w.write(0, sc.pos)  # velocities required


@pytest.mark.gpu
def test_recorded_run_is_reproduced(tmp_path):
    from pbf_b200 import Solver
    sc = _scene()
    path = os.path.join(tmp_path, "run.pbft")
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    s.upload(sc.pos, sc.vel)
    assert record(s, path, sc.para, sc.grid_space, sc.boundary, substeps=6, every=2) == 4
    r = TrajectoryReader(path)
    assert [f[0] for f in r] == [0, 2, 4, 6]
    t = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    t.upload(sc.pos, sc.vel)
    for k in range(1, 4):
        t.step(2)
        p, v = t.download()
        assert np.array_equal(p, r[k][1]) and np.array_equal(v, r[k][2])
