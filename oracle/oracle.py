"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (pbf_oracle.cpp)
and to the reference checkers built from the reference sources (oracle/_ref/).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed reference CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REFCPU_SO = os.path.join(HERE, "_ref", "libpbfref_cpu.so")
REFGPU_SO = os.path.join(HERE, "_ref", "libpbfref_gpu.so")

F = {"x": 0, "v": 1, "xold": 2, "xpred": 3, "lambda": 4, "rho": 5, "dp": 6, "curl": 7, "vort": 8, "visc": 9,
     "cell": 10, "cnt": 11, "start": 12, "end": 13, "sorted": 14, "ncnt": 15, "nbr": 16, "perm": 17, "dpmag": 18}
VEC3 = {"x", "v", "xold", "xpred", "dp", "curl", "vort", "visc"}
SCALAR = {"lambda", "rho", "dpmag"}
PER_CELL = {"cnt", "start", "end"}


class OracleParams(C.Structure):
    _fields_ = [
        ("h", C.c_float), ("restRho", C.c_float), ("epsilon", C.c_float), ("k", C.c_float), ("n", C.c_float),
        ("deltaq", C.c_float), ("c", C.c_float), ("dt", C.c_float), ("vort_eps", C.c_float),
        ("iterations", C.c_int), ("gravity", C.c_float * 3), ("grid_min", C.c_float * 3), ("dims", C.c_int * 3),
        ("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("wall_jitter", C.c_float), ("grad_rmin", C.c_float),
        ("max_nbr", C.c_int), ("formulation", C.c_int), ("arith", C.c_int), ("cell_order", C.c_int),
        ("reorder", C.c_int), ("flags", C.c_int), ("scorr_scale", C.c_float), ("sphere", C.c_float * 4),
        ("wall_jitter_d", C.c_double), ("cell_scale", C.c_float), ("lanes", C.c_int),
    ]


def ensure_built() -> None:
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


_olib = None


def olib() -> C.CDLL:
    global _olib
    if _olib is None:
        ensure_built()
        L = C.CDLL(ORACLE_SO)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(OracleParams), C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_substep.argtypes = [C.c_void_p]
        L.oracle_set_params.argtypes = [C.c_void_p, C.POINTER(OracleParams)]
        L.oracle_substep_adaptive.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        L.oracle_build_only.argtypes = [C.c_void_p]
        L.oracle_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_ncells.argtypes = [C.c_void_p]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_det_sin.restype = C.c_float
        L.oracle_det_sin.argtypes = [C.c_float]
        L.oracle_rsqrt.restype = C.c_float
        L.oracle_rsqrt.argtypes = [C.c_float]
        L.oracle_density_error.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.c_void_p]
        _olib = L
    return _olib


def params_from(para, grid_space, boundary, *, gravity=(0.0, -49.0, 0.0), dims=(64, 64, 64), formulation=0,
                arith=1, cell_order=0, reorder=1, flags=0, scorr_scale=1.0, wall_jitter=None, grad_rmin=0.01,
                max_nbr=63, sphere=(0, 0, 0, 0), cell_scale=1.0, iterations=None, lanes=2) -> OracleParams:
    """Oracle parameters from a SolverParameter-like object and the two AABBs.
    lanes: pair lanes per particle of the product arithmetic (the library's
    pair_lanes, default 2)."""
    p = OracleParams()
    for f in ("h", "restRho", "epsilon", "k", "n", "deltaq", "c", "dt"):
        setattr(p, f, float(getattr(para, f)))
    p.vort_eps = float(para.vorticityConfinementEpilon)
    p.iterations = int(para.iterations if iterations is None else iterations)
    for a in range(3):
        p.gravity[a] = gravity[a]
        p.grid_min[a] = grid_space[a]
        p.dims[a] = dims[a]
        p.bmin[a] = boundary[a]
        p.bmax[a] = boundary[3 + a]
    if wall_jitter is None:
        wall_jitter = 0.01 if formulation == 0 else 0.02
    p.wall_jitter = wall_jitter
    p.wall_jitter_d = 0.01 if formulation == 0 else float(np.float32(wall_jitter))
    p.grad_rmin = grad_rmin
    p.max_nbr = max_nbr
    p.formulation = formulation
    p.arith = arith
    p.cell_order = cell_order
    p.reorder = reorder
    p.flags = flags
    p.scorr_scale = scorr_scale
    for a in range(4):
        p.sphere[a] = sphere[a]
    p.cell_scale = cell_scale
    p.lanes = lanes
    return p


def params_for_scene(scene, ext=None, **kw) -> OracleParams:
    """Oracle parameters matching a pbf_b200 Scene (+ ext overrides) in product arithmetic."""
    ov = dict(scene.ext_overrides)
    if ext:
        ov.update(ext)
    return params_from(scene.para, scene.grid_space, scene.boundary, gravity=ov.get("gravity", (0, -49, 0)),
                       dims=ov.get("grid_dims", (64, 64, 64)), flags=ov.get("flags", 0),
                       scorr_scale=ov.get("scorr_scale", 1.0), wall_jitter=ov.get("wall_jitter", 0.01),
                       grad_rmin=ov.get("grad_rmin", 0.01), max_nbr=ov.get("max_neighbors", 63),
                       sphere=ov.get("sphere", (0, 0, 0, 0)), cell_scale=ov.get("cell_scale", 1.0),
                       cell_order=ov.get("cell_order", 0), lanes=kw.pop("lanes", ov.get("pair_lanes", 0) or 2), **kw)


class Oracle:
    """One oracle simulation (float or double)."""

    def __init__(self, params: OracleParams, pos: np.ndarray, vel: np.ndarray, precision: int = 32):
        self.n = int(pos.shape[0])
        self.params = params
        p = np.ascontiguousarray(pos, np.float32)
        v = np.ascontiguousarray(vel, np.float32)
        self._h = olib().oracle_create(C.byref(params), precision, self.n, p.ctypes.data, v.ctypes.data)
        if not self._h:
            raise ValueError("oracle_create rejected the parameters")
        self.ncells = olib().oracle_ncells(self._h)

    def substep(self, count: int = 1) -> None:
        for _ in range(count):
            olib().oracle_substep(self._h)

    def set_params(self, params: OracleParams) -> None:
        """New parameter values for the following substeps (same grid and cap)."""
        if olib().oracle_set_params(self._h, C.byref(params)) != 0:
            raise ValueError("oracle_set_params: the grid or the neighbour cap changed")
        self.params = params

    def substep_adaptive(self, tol: float, min_iterations: int, max_iterations: int) -> int:
        """One adaptive substep of the CUDA library (ext.adaptive): corrections until
        the lambda pass measures a max one-sided density error <= tol, at least
        min_iterations (>= 1) and at most max_iterations; returns the count."""
        return int(olib().oracle_substep_adaptive(self._h, float(tol), int(min_iterations), int(max_iterations)))

    def build_only(self) -> None:
        olib().oracle_build_only(self._h)

    def get(self, name: str) -> np.ndarray:
        fid = F[name]
        if name in VEC3:
            out = np.empty((self.n, 3), np.float64)
            olib().oracle_get(self._h, fid, out.ctypes.data, None)
        elif name in SCALAR:
            out = np.empty(self.n, np.float64)
            olib().oracle_get(self._h, fid, out.ctypes.data, None)
        else:
            size = self.ncells if name in PER_CELL else (self.n * self.params.max_nbr if name == "nbr" else self.n)
            out = np.empty(size, np.int32)
            olib().oracle_get(self._h, fid, None, out.ctypes.data)
        return out

    def close(self) -> None:
        if self._h:
            olib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def det_sin(a: float) -> float:
    return olib().oracle_det_sin(a)


def rsqrt(x: float) -> float:
    return olib().oracle_rsqrt(x)


def density_error(pos: np.ndarray, h: float, rho0: float, per_particle: bool = False):
    """FP64 one-sided density error over all pairs within h: (max, mean[, per-particle])."""
    p = np.ascontiguousarray(pos, np.float32)
    n = p.shape[0]
    mx, mean = C.c_double(), C.c_double()
    err = np.empty(n, np.float64) if per_particle else None
    olib().oracle_density_error(n, p.ctypes.data, h, rho0, C.byref(mx), C.byref(mean),
                                None if err is None else err.ctypes.data)
    return (mx.value, mean.value, err) if per_particle else (mx.value, mean.value)


# ---- reference CPU solver (src/solver.cpp, built as-is) ---------------------
_rlib = None


def refcpu_available() -> bool:
    return os.path.exists(REFCPU_SO)


def rlib() -> C.CDLL:
    global _rlib
    if _rlib is None:
        L = C.CDLL(REFCPU_SO)
        L.refcpu_create.restype = C.c_void_p
        L.refcpu_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.refcpu_set_threads.argtypes = [C.c_int]
        L.refcpu_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.refcpu_build.argtypes = [C.c_void_p, C.c_void_p]
        L.refcpu_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.refcpu_ncells.argtypes = [C.c_void_p]
        L.refcpu_destroy.argtypes = [C.c_void_p]
        _rlib = L
    return _rlib


REF_FIELDS = {"lambda": 0, "dp": 1, "curl": 2, "vort": 3, "visc": 4, "xold": 5, "cell": 6, "start": 7, "end": 8,
              "sorted": 9, "ncnt": 10, "nbr": 11}


class RefCpu:
    """The reference's own PBFSolver (include/solver.h:83-222)."""

    def __init__(self, para, box, dims=(64, 64, 64)):
        self.n = int(para.nParticles)
        self._para = para
        b = np.ascontiguousarray(box, np.float32)
        d = np.ascontiguousarray(dims, np.int32)
        self._h = rlib().refcpu_create(C.byref(para), b.ctypes.data, d.ctypes.data)
        self.ncells = rlib().refcpu_ncells(self._h)

    def set_threads(self, t: int) -> None:
        rlib().refcpu_set_threads(t)

    def solve(self, pos: np.ndarray, vel: np.ndarray, substeps: int = 1, quiet: bool = True):
        p = np.ascontiguousarray(pos, np.float32).copy()
        v = np.ascontiguousarray(vel, np.float32).copy()
        rlib().refcpu_solve(self._h, p.ctypes.data, v.ctypes.data, substeps, 1 if quiet else 0)
        return p, v

    def build(self, pos: np.ndarray) -> None:
        p = np.ascontiguousarray(pos, np.float32)
        rlib().refcpu_build(self._h, p.ctypes.data)

    def get(self, name: str) -> np.ndarray:
        fid = REF_FIELDS[name]
        if name in ("dp", "curl", "vort", "visc", "xold"):
            out = np.empty((self.n, 3), np.float64)
            rlib().refcpu_get(self._h, fid, out.ctypes.data, None)
        elif name == "lambda":
            out = np.empty(self.n, np.float64)
            rlib().refcpu_get(self._h, fid, out.ctypes.data, None)
        else:
            size = self.ncells if name in ("start", "end") else (self.n * 63 if name == "nbr" else self.n)
            out = np.empty(size, np.int32)
            rlib().refcpu_get(self._h, fid, None, out.ctypes.data)
        return out

    def close(self) -> None:
        if self._h:
            rlib().refcpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- reference CUDA solver (kernels/cudaPBF*.cu, built as-is) ---------------
def refgpu_available() -> bool:
    return os.path.exists(REFGPU_SO)


def refgpu_run(para, grid_space, boundary, pos, vel, substeps: int = 1) -> dict:
    """Runs the reference CUDA solver (64^3 grid) and returns all SolverData arrays."""
    L = C.CDLL(REFGPU_SO)
    L.refgpu_run.argtypes = [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 12
    n = int(para.nParticles)
    out = {k: np.zeros((n, 3), np.float32) for k in ("x", "v", "xold", "dp", "curl", "vort", "visc")}
    out["lambda"] = np.zeros(n, np.float32)
    out["nbr"] = np.zeros((n, 64), np.int32)
    out["grid"] = np.zeros((64 ** 3, 2), np.uint32)
    out["sorted"] = np.zeros(n, np.int32)
    out["prefix"] = np.zeros(64 ** 3, np.int32)
    gs = np.ascontiguousarray(grid_space, np.float32)
    bd = np.ascontiguousarray(boundary, np.float32)
    p = np.ascontiguousarray(pos, np.float32)
    v = np.ascontiguousarray(vel, np.float32)
    rc = L.refgpu_run(C.byref(para), gs.ctypes.data, bd.ctypes.data, p.ctypes.data, v.ctypes.data, substeps,
                      out["x"].ctypes.data, out["v"].ctypes.data, out["xold"].ctypes.data, out["lambda"].ctypes.data,
                      out["dp"].ctypes.data, out["curl"].ctypes.data, out["vort"].ctypes.data,
                      out["visc"].ctypes.data, out["nbr"].ctypes.data, out["grid"].ctypes.data,
                      out["sorted"].ctypes.data, out["prefix"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"refgpu_run failed: {rc}")
    return out
