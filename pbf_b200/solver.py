"""Host-side mirror of the reference solver interface over the C ABI.

Reference interfaces mirrored:
  * PBFSolver(para, box) / solve(Particle*)        include/solver.h:86-111
  * initCUDASolverDataBuffer / cudaPBFSolve /
    freeCUDASolverDataBuffer                       kernels/cudaPBF.h:8-12
Same names, argument meaning and error behaviour (errors raise PBFError with the
C status code instead of exiting the process).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import ExtParams, PBFError, SolverParameter, Stats, check, lib


def make_parameter(**kw) -> SolverParameter:
    """SolverParameter with invDt filled from dt when not given."""
    p = SolverParameter()
    for k, v in kw.items():
        setattr(p, k, v)
    if "invDt" not in kw and p.dt:
        p.invDt = np.float32(1.0) / np.float32(p.dt)
    return p


def default_ext(**overrides) -> ExtParams:
    e = ExtParams()
    lib().pbf_ext_params_default(C.byref(e))
    for k, v in overrides.items():
        if k in ("gravity", "grid_dims", "sphere"):
            arr = getattr(e, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(e, k, v)
    return e


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)  # torch.cuda.Stream


def _host_ptr(a, n: int, writable: bool = False) -> int:
    """Address of an n x 3 float32 C-contiguous host array (numpy or CPU tensor)."""
    if hasattr(a, "data_ptr"):  # torch tensor
        if a.is_cuda or a.dtype.itemsize != 4 or not a.is_contiguous() or a.numel() != 3 * n:
            raise ValueError("expected a contiguous float32 host tensor of n x 3")
        return a.data_ptr()
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous and a.size == 3 * n):
        raise ValueError("expected a C-contiguous float32 array of n x 3")
    if writable and not a.flags.writeable:
        raise ValueError("output array is read-only")
    return a.ctypes.data


def _f6(b: Sequence[float]):
    a = (C.c_float * 6)(*[float(x) for x in b])
    return a


class Solver:
    """One PBF scene on the GPU (a pbf_solver handle)."""

    def __init__(self, para: SolverParameter, grid_space: Sequence[float], boundary: Sequence[float],
                 ext: Optional[ExtParams] = None):
        self.para = para
        self.ext = ext if ext is not None else default_ext()
        self.n = int(para.nParticles)
        h = C.c_void_p()
        check(lib().pbf_create(C.byref(para), _f6(grid_space), _f6(boundary), C.byref(self.ext), C.byref(h)))
        self._h = h
        nc, st, mn = C.c_int(), C.c_int(), C.c_int()
        check(lib().pbf_get_layout(h, C.byref(nc), C.byref(st), C.byref(mn)))
        self.ncells, self.stride, self.max_neighbors = nc.value, st.value, mn.value

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pbf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- data -----------------------------------------------------------------
    def upload(self, pos: np.ndarray, vel: np.ndarray) -> None:
        p = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1)
        v = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1)
        if p.size != 3 * self.n or v.size != 3 * self.n:
            raise PBFError(_lib.PBF_ERR_INVALID, f"expected {self.n} xyz positions and velocities")
        check(lib().pbf_upload(self._h, p.ctypes.data, v.ctypes.data, self.n))

    def upload_device(self, d_pos, d_vel, stream=None) -> None:
        """d_pos / d_vel: CUDA tensors (float32, n x 3 contiguous) or raw device pointers."""
        pp = d_pos if isinstance(d_pos, int) else d_pos.data_ptr()
        vp = d_vel if isinstance(d_vel, int) else d_vel.data_ptr()
        check(lib().pbf_upload_device(self._h, pp, vp, self.n, _stream_handle(stream)))

    def bind_position(self, d_pos) -> None:
        ptr = None if d_pos is None else (d_pos if isinstance(d_pos, int) else d_pos.data_ptr())
        check(lib().pbf_bind_position(self._h, ptr))

    def step(self, substeps: int = 1, stream=None) -> None:
        check(lib().pbf_step(self._h, int(substeps), _stream_handle(stream)))

    def set_parameter(self, para: SolverParameter) -> None:
        """New SolverParameter values for the following substeps (pbf_set_parameter);
        nParticles must stay the same."""
        check(lib().pbf_set_parameter(self._h, C.byref(para)))
        self.para = para

    def build_grid(self, stream=None) -> None:
        check(lib().pbf_build_grid(self._h, _stream_handle(stream)))

    def download(self):
        pos = np.empty((self.n, 3), np.float32)
        vel = np.empty((self.n, 3), np.float32)
        check(lib().pbf_download(self._h, pos.ctypes.data, vel.ctypes.data))
        return pos, vel

    def download_device(self, d_pos=None, d_vel=None, stream=None) -> None:
        pp = None if d_pos is None else (d_pos if isinstance(d_pos, int) else d_pos.data_ptr())
        vp = None if d_vel is None else (d_vel if isinstance(d_vel, int) else d_vel.data_ptr())
        check(lib().pbf_download_device(self._h, pp, vp, _stream_handle(stream)))

    def step_host(self, pos, vel, pos_out, substeps: int = 1, stream=None) -> None:
        """One asynchronous frame from and to host memory (pbf_step_host): pos, vel
        and pos_out are n x 3 float32 host arrays (numpy or CPU tensors; pinned
        memory lets the copies overlap). They must stay untouched until
        host_fence(stream) has been called and the stream synchronised."""
        check(lib().pbf_step_host(self._h, _host_ptr(pos, self.n), _host_ptr(vel, self.n),
                                  _host_ptr(pos_out, self.n, writable=True), int(substeps),
                                  _stream_handle(stream)))

    def host_fence(self, stream=None) -> None:
        """Makes `stream` wait for every copy issued by step_host so far."""
        check(lib().pbf_host_fence(self._h, _stream_handle(stream)))

    def resize(self, n: int) -> None:
        """Particle count of a single-scene solver (<= the count it was created
        with); needs a new upload before the next step."""
        check(lib().pbf_resize(self._h, int(n)))
        self.n = int(n)

    def download_sorted_device(self, pos=None, vel=None, ids=None, key=None, rank=None, stream=None) -> None:
        """The state after the last step in slot order into device tensors: n x 3
        float32 pos / vel, int32 ids (index in the uploaded order), key (cell the
        slot was sorted into) and rank (slot within that cell); any may be None."""
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        check(lib().pbf_download_sorted_device(self._h, ptr(pos), ptr(vel), ptr(ids), ptr(key), ptr(rank),
                                               _stream_handle(stream)))

    def stats(self, raise_on_error: bool = True) -> dict:
        st = Stats()
        rc = lib().pbf_get_stats(self._h, C.byref(st))
        if raise_on_error:
            check(rc)
        return {k: getattr(st, k) for k, _ in Stats._fields_}

    def stage_times(self) -> dict:
        """Per-stage milliseconds of the last substep (needs ext.profile = 1)."""
        ms = (C.c_float * len(_lib.STAGES))()
        check(lib().pbf_stage_times(self._h, ms, len(_lib.STAGES)))
        return {name: float(ms[i]) for i, name in enumerate(_lib.STAGES)}

    def kernel_count(self) -> int:
        """Kernel launches per substep (kernel nodes of the substep graph)."""
        rc = lib().pbf_graph_kernel_count(self._h)
        if rc < 0:
            check(rc)
        return rc

    def measure_density_error(self, stream=None):
        """(max, mean) one-sided density error of the current state."""
        mx, mean = C.c_double(), C.c_double()
        check(lib().pbf_measure_density_error(self._h, C.byref(mx), C.byref(mean), _stream_handle(stream)))
        return mx.value, mean.value

    def fetch(self, name: str) -> np.ndarray:
        """Internal array in cell-sorted slot order."""
        fid = _lib.FIELD[name]
        nbytes = lib().pbf_field_bytes(self._h, fid)
        if name in _lib.FLOAT4_FIELDS:
            out = np.empty((self.n, 4), np.float32)
        elif name == "features":
            out = np.empty((self.n, 12), np.float32)
        elif name in _lib.FLOAT_FIELDS:
            out = np.empty(self.n, np.float32)
        else:
            out = np.empty(nbytes // 4, np.int32)
        assert out.nbytes == nbytes, (name, out.nbytes, nbytes)
        check(lib().pbf_fetch(self._h, fid, out.ctypes.data, nbytes))
        return out

    def fetch_original(self, name: str) -> np.ndarray:
        """A per-particle field mapped back to original particle order."""
        a = self.fetch(name)
        perm = self.fetch("perm")
        out = np.empty_like(a)
        out[perm] = a
        return out

    def neighbor_lists(self) -> list:
        """Neighbour slot lists (slot order) as Python lists, for tests."""
        nbr = self.fetch("nbr").reshape(self.max_neighbors, self.stride)
        cnt = self.fetch("ncnt")
        return [nbr[: cnt[k], k].tolist() for k in range(self.n)]


class BatchSolver(Solver):
    """Many independent scenes in one handle (pbf_create_batch): every phase of
    a substep is one launch over all scenes; positions and velocities are
    concatenated in scene order. All scenes share the SolverParameter values and
    the ext flags; each has its own grid, wall box and obstacle."""

    def __init__(self, para: SolverParameter, scenes: Sequence[dict], ext: Optional[ExtParams] = None):
        """scenes: dicts with grid_space, boundary, grid_dims, nparticles, optional sphere."""
        self.para = para
        self.ext = ext if ext is not None else default_ext()
        self.n = int(para.nParticles)
        descs = (_lib.SceneDesc * len(scenes))()
        for i, d in enumerate(scenes):
            for a in range(6):
                descs[i].grid_space[a] = float(d["grid_space"][a])
                descs[i].boundary[a] = float(d["boundary"][a])
            for a in range(3):
                descs[i].grid_dims[a] = int(d["grid_dims"][a])
            descs[i].nparticles = int(d["nparticles"])
            for a, v in enumerate(d.get("sphere", (0.0, 0.0, 0.0, 0.0))):
                descs[i].sphere[a] = float(v)
        h = C.c_void_p()
        check(lib().pbf_create_batch(C.byref(para), len(scenes), descs, C.byref(self.ext), C.byref(h)))
        self._h = h
        nc, st, mn = C.c_int(), C.c_int(), C.c_int()
        check(lib().pbf_get_layout(h, C.byref(nc), C.byref(st), C.byref(mn)))
        self.ncells, self.stride, self.max_neighbors = nc.value, st.value, mn.value
        self.nscenes = len(scenes)

    def scene_layout(self, i: int) -> dict:
        cb, nc, pb, pc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().pbf_get_scene_layout(self._h, i, C.byref(cb), C.byref(nc), C.byref(pb), C.byref(pc)))
        return {"cell_base": cb.value, "ncells": nc.value, "pbase": pb.value, "pcount": pc.value}


class PBFSolver:
    """The reference CPU solver's interface (include/solver.h:86-111) on the GPU
    step: construct with the parameters and box, then solve(particles) advances
    an array of particles (n x 6: position xyz, velocity xyz) by one substep in
    place. The wall is the box shrunk by para.radius (include/solver.h:97)."""

    def __init__(self, para: SolverParameter, box: Sequence[float], ext: Optional[ExtParams] = None,
                 grid_space: Optional[Sequence[float]] = None):
        r = float(para.radius)
        bd = [box[0] + r, box[1] + r, box[2] + r, box[3] - r, box[4] - r, box[5] - r]
        self.solver = Solver(para, grid_space if grid_space is not None else box, bd, ext)
        self._uploaded = False

    def solve(self, particles: np.ndarray) -> None:
        if particles.dtype != np.float32 or particles.shape != (self.solver.n, 6):
            raise PBFError(_lib.PBF_ERR_INVALID, "particles must be float32 (n, 6)")
        self.solver.upload(particles[:, :3], particles[:, 3:])
        self.solver.step(1)
        pos, vel = self.solver.download()
        particles[:, :3] = pos
        particles[:, 3:] = vel


# -- the three entry points of kernels/cudaPBF.h:8-12 --------------------------
def initCUDASolverDataBuffer(position: np.ndarray, velocity: np.ndarray, para: SolverParameter,
                             gridSpace: Sequence[float], boundary: Sequence[float],
                             ext: Optional[ExtParams] = None) -> Solver:
    s = Solver(para, gridSpace, boundary, ext)
    s.upload(position, velocity)
    return s


def cudaPBFSolve(data: Solver, para: Optional[SolverParameter] = None) -> None:
    """One substep; like the reference (kernels/cudaPBF.cu:50-115) it takes the
    parameters of this call, so changed values apply from this substep on."""
    if para is not None:
        data.set_parameter(para)
    data.step(1)


def freeCUDASolverDataBuffer(data: Solver) -> None:
    data.close()
