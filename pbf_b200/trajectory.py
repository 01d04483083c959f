"""Trajectory files: particle positions (and velocities) of a run, frame by frame.

The reference has no I/O; this is the format the library uses to keep runs for
regression fixtures and for training the learned warm start offline.

Layout (little-endian):

  header, 256 bytes
    0   8  magic b"PBFTRAJ1"
    8   4  u32 format version (1)
   12   4  u32 particle count n
   16   4  u32 flags: bit 0 = frames carry velocities
   20   4  u32 reserved (0)
   24   8  u64 frame count (written when the file is closed; a reader also
           derives it from the file size and uses the smaller of the two)
   32  52  SolverParameter of the run (the reference's struct, include/solverBase.h:16-40)
   84  24  grid space: pMin xyz, pMax xyz (float32)
  108  24  boundary:   pMin xyz, pMax xyz (float32)
  132 124  zero
  frames, each:
    i64 substep index, then float32 positions [n][3], then (flag) float32 velocities [n][3]

Positions and velocities are in the caller's particle order (the order given to
upload), not the solver's internal cell order.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from typing import Iterator, Optional, Sequence, Tuple

import numpy as np

from ._lib import SolverParameter

MAGIC = b"PBFTRAJ1"
VERSION = 1
HEADER_BYTES = 256
FLAG_VELOCITY = 1
_HEAD = struct.Struct("<8sIIIIQ")


def _frame_bytes(n: int, flags: int) -> int:
    return 8 + 12 * n * (2 if flags & FLAG_VELOCITY else 1)


class TrajectoryWriter:
    """Appends frames to a new trajectory file."""

    def __init__(self, path: str, para: SolverParameter, grid_space: Sequence[float], boundary: Sequence[float],
                 n: int, velocities: bool = True):
        if n <= 0:
            raise ValueError("particle count must be positive")
        self.path = path
        self.n = int(n)
        self.flags = FLAG_VELOCITY if velocities else 0
        self.frames = 0
        self._f = open(path, "wb")
        head = bytearray(HEADER_BYTES)
        head[0:_HEAD.size] = _HEAD.pack(MAGIC, VERSION, self.n, self.flags, 0, 0)
        raw = bytes(para)
        if len(raw) != 52:
            raise ValueError("SolverParameter must be 52 bytes")
        head[32:84] = raw
        head[84:108] = np.asarray(grid_space, np.float32).reshape(6).tobytes()
        head[108:132] = np.asarray(boundary, np.float32).reshape(6).tobytes()
        self._f.write(head)

    def write(self, substep: int, pos: np.ndarray, vel: Optional[np.ndarray] = None) -> None:
        p = np.ascontiguousarray(pos, np.float32)
        if p.shape != (self.n, 3):
            raise ValueError(f"positions must be ({self.n}, 3)")
        self._f.write(struct.pack("<q", int(substep)))
        self._f.write(p.tobytes())
        if self.flags & FLAG_VELOCITY:
            if vel is None:
                raise ValueError("this trajectory stores velocities")
            v = np.ascontiguousarray(vel, np.float32)
            if v.shape != (self.n, 3):
                raise ValueError(f"velocities must be ({self.n}, 3)")
            self._f.write(v.tobytes())
        self.frames += 1

    def close(self) -> None:
        if self._f is None:
            return
        self._f.seek(24)
        self._f.write(struct.pack("<Q", self.frames))
        self._f.close()
        self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class TrajectoryReader:
    """Random access to the frames of a trajectory file (memory-mapped)."""

    def __init__(self, path: str):
        size = os.path.getsize(path)
        if size < HEADER_BYTES:
            raise ValueError(f"{path}: not a trajectory file (too short)")
        with open(path, "rb") as f:
            head = f.read(HEADER_BYTES)
        magic, version, n, flags, _, frames = _HEAD.unpack_from(head, 0)
        if magic != MAGIC:
            raise ValueError(f"{path}: not a trajectory file (bad magic)")
        if version != VERSION:
            raise ValueError(f"{path}: unsupported trajectory version {version}")
        self.path = path
        self.n = n
        self.flags = flags
        self.para = SolverParameter.from_buffer_copy(head[32:84])
        self.grid_space = np.frombuffer(head[84:108], np.float32).copy()
        self.boundary = np.frombuffer(head[108:132], np.float32).copy()
        fb = _frame_bytes(n, flags)
        complete = (size - HEADER_BYTES) // fb
        # a file whose writer did not close it still yields its complete frames
        self.nframes = int(min(frames, complete)) if frames else int(complete)
        self._mm = np.memmap(path, np.uint8, mode="r", offset=HEADER_BYTES, shape=(self.nframes * fb,)) \
            if self.nframes else None
        self._fb = fb

    def __len__(self) -> int:
        return self.nframes

    def __getitem__(self, k: int) -> Tuple[int, np.ndarray, Optional[np.ndarray]]:
        """(substep, positions [n, 3], velocities [n, 3] or None) of frame k."""
        if k < 0:
            k += self.nframes
        if not 0 <= k < self.nframes:
            raise IndexError(k)
        base = k * self._fb
        rec = self._mm[base:base + self._fb]
        step = int(np.frombuffer(rec[:8].tobytes(), "<i8")[0])
        pos = np.frombuffer(rec[8:8 + 12 * self.n].tobytes(), np.float32).reshape(self.n, 3)
        vel = None
        if self.flags & FLAG_VELOCITY:
            vel = np.frombuffer(rec[8 + 12 * self.n:].tobytes(), np.float32).reshape(self.n, 3)
        return step, pos, vel

    def __iter__(self) -> Iterator[Tuple[int, np.ndarray, Optional[np.ndarray]]]:
        for k in range(self.nframes):
            yield self[k]


def record(solver, path: str, para: SolverParameter, grid_space: Sequence[float], boundary: Sequence[float],
           substeps: int, every: int = 1, velocities: bool = True, include_start: bool = True) -> int:
    """Runs `solver` (already uploaded) for `substeps` substeps and writes a frame
    every `every` substeps (and the starting state when include_start); returns
    the number of frames written."""
    if every <= 0:
        raise ValueError("every must be positive")
    with TrajectoryWriter(path, para, grid_space, boundary, solver.n, velocities) as w:
        if include_start:
            p, v = solver.download()
            w.write(0, p, v)
        done = 0
        while done < substeps:
            k = min(every, substeps - done)
            solver.step(k)
            done += k
            p, v = solver.download()
            w.write(done, p, v)
        return w.frames
