"""The C-ABI library (CPU tests: load, exports, layouts, host-side validation)."""
import ctypes as C
import os
import re

import pytest

from pbf_b200 import _lib
from pbf_b200._lib import ExtParams, SolverParameter, Stats, lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pbf.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pbf_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_function_is_exported_and_bound():
    L = lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), f"{name} declared in include/pbf.h but not exported"
    assert set(names) <= set(_lib.declared_symbols()), set(names) - set(_lib.declared_symbols())


def test_struct_layouts_match_the_c_side():
    L = lib()
    assert L.pbf_struct_size(0) == C.sizeof(SolverParameter) == 52
    assert L.pbf_struct_size(1) == C.sizeof(ExtParams)
    assert L.pbf_struct_size(2) == C.sizeof(Stats)
    from pbf_b200._lib import Camera
    assert L.pbf_struct_size(3) == C.sizeof(Camera)
    assert L.pbf_abi_version() == 1


def test_defaults_are_the_reference_constants():
    e = ExtParams()
    lib().pbf_ext_params_default(C.byref(e))
    assert list(e.gravity) == [0.0, -49.0, 0.0]  # kernels/cudaPBFSolver.cu:9
    assert list(e.grid_dims) == [64, 64, 64]  # include/solverBase.h:10-12
    assert e.max_neighbors == 63  # include/solverBase.h:6
    assert abs(e.wall_jitter - 0.01) < 1e-9  # include/solverBase.h:5
    assert abs(e.grad_rmin - 0.01) < 1e-9  # kernels/cudaPBFSolver.cuh:107
    assert e.cell_scale == 1.0 and e.scorr_scale == 1.0 and e.flags == 0


def _create(para=None, ext=None, gs=(0, 0, 0, 4, 2, 2), bd=(0.03, 0.03, 0.03, 3.97, 1.97, 1.97)):
    from pbf_b200 import make_parameter
    p = para or make_parameter(h=0.1, nParticles=100, restRho=6378.0, epsilon=600.0, k=0.1, n=4.0, deltaq=0.02,
                               c=0.01, dt=1 / 120, iterations=4, vorticityConfinementEpilon=0.0005, radius=0.03)
    e = ext or ExtParams()
    if ext is None:
        lib().pbf_ext_params_default(C.byref(e))
    h = C.c_void_p()
    rc = lib().pbf_create(C.byref(p), (C.c_float * 6)(*gs), (C.c_float * 6)(*bd), C.byref(e), C.byref(h))
    return rc, h, p, e


@pytest.mark.parametrize("field,value", [("nParticles", 0), ("h", 0.0), ("restRho", -1.0), ("dt", 0.0),
                                          ("deltaq", 0.5), ("iterations", -1), ("iterations", 65),
                                          ("epsilon", float("nan"))])
def test_create_rejects_bad_parameters_without_touching_the_gpu(field, value):
    rc, h, p, e = _create()
    if rc == 0:
        lib().pbf_destroy(h)
    from pbf_b200 import make_parameter
    p = make_parameter(h=0.1, nParticles=100, restRho=6378.0, epsilon=600.0, k=0.1, n=4.0, deltaq=0.02, c=0.01,
                       dt=1 / 120, iterations=4, vorticityConfinementEpilon=0.0005, radius=0.03)
    setattr(p, field, value)
    rc, h, _, _ = _create(para=p)
    assert rc == _lib.PBF_ERR_INVALID
    assert lib().pbf_last_error()


@pytest.mark.parametrize("field,value", [("max_neighbors", 0), ("max_neighbors", 128), ("cell_scale", 0.2),
                                          ("cell_order", 2), ("max_iterations", 0), ("max_iterations", 65)])
def test_create_rejects_bad_extensions(field, value):
    e = ExtParams()
    lib().pbf_ext_params_default(C.byref(e))
    setattr(e, field, value)
    rc, h, _, _ = _create(ext=e)
    assert rc == _lib.PBF_ERR_INVALID


@pytest.mark.parametrize("m,tile", [(1, 8192), (8192, 8192), (8193, 8192), (1 << 22, 8192),
                                    ((1 << 22) + 1, 16384), (16_777_216, 16384)])
def test_scan_workspace_holds_one_status_word_per_tile(m, tile):
    """The scan's workspace: one 8-byte status word per tile, the tile counter
    and the error word; tiles of 8,192 counts up to 2^22 counts, of 16,384 above
    (host arithmetic only, no GPU)."""
    tiles = -(-m // tile)
    assert lib().pbf_scan_workspace_bytes(m) == tiles * 8 + 16 + 16


def test_null_handles_are_errors_not_crashes():
    L = lib()
    assert L.pbf_step(None, 1, None) == _lib.PBF_ERR_INVALID
    assert L.pbf_upload(None, None, None, 0) == _lib.PBF_ERR_INVALID
    assert L.pbf_download(None, None, None) == _lib.PBF_ERR_INVALID
    assert L.pbf_destroy(None) == _lib.PBF_OK
    st = Stats()
    assert L.pbf_get_stats(None, C.byref(st)) == _lib.PBF_ERR_INVALID
    assert L.pbf_scan_exclusive_i32(None, None, 4, None, 0, None) == _lib.PBF_ERR_INVALID


def test_test_hooks_validate_on_the_host():
    """The failure-injection hooks reject bad arguments before touching a GPU."""
    L = lib()
    bits = C.c_int(0)
    assert L.pbf_debug_expire_wait(2, C.byref(bits)) == _lib.PBF_ERR_INVALID
    assert L.pbf_debug_expire_wait(0, None) == _lib.PBF_ERR_INVALID
    assert L.pbf_debug_fail_staging_alloc(-1) == _lib.PBF_ERR_INVALID
    assert L.pbf_debug_fail_staging_alloc(0) == _lib.PBF_OK


@pytest.mark.parametrize("m", [(1 << 30) + 1, 2**31 - 1])
def test_scan_rejects_counts_beyond_its_limit(m):
    """Counts above PBF_SCAN_MAX_COUNT (2^30) are refused on the host: no
    workspace size, PBF_ERR_INVALID from the scan (tile arithmetic in 64 bits)."""
    L = lib()
    assert L.pbf_scan_workspace_bytes(m) == 0
    assert L.pbf_scan_exclusive_i32(C.c_void_p(16), C.c_void_p(16), m, C.c_void_p(16), 1 << 20, None) == \
        _lib.PBF_ERR_INVALID
    tiles = -(-(1 << 30) // 16384)
    assert L.pbf_scan_workspace_bytes(1 << 30) == tiles * 8 + 16 + 16


def test_set_parameter_validates_on_the_host():
    L = lib()
    p = SolverParameter()
    assert L.pbf_set_parameter(None, C.byref(p)) == _lib.PBF_ERR_INVALID


from pbf_b200.build import reference_dir  # noqa: E402

REF = reference_dir()


@pytest.mark.skipif(not REF, reason="reference headers not present")
def test_reference_shim_exports_the_reference_symbols(tmp_path):
    """reference_shim.cpp compiles against the reference's own headers and
    defines the same (mangled) functions the reference's kernels/cudaPBF.cu does."""
    import subprocess
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    obj = tmp_path / "shim.o"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-c", f"-I{REF}/include", f"-I{REF}/ext", f"-I{REF}/ext/glfw/include",
                    f"-I{repo}/include", os.path.join(repo, "pbf_b200", "csrc", "reference_shim.cpp"), "-o",
                    str(obj)], check=True)
    ours = subprocess.run(["nm", "-g", "--defined-only", str(obj)], capture_output=True, text=True).stdout
    want = ["cudaPBFSolve", "initCUDASolverDataBuffer", "freeCUDASolverDataBuffer"]
    ref_so = os.path.join(repo, "oracle", "_ref", "libpbfref_gpu.so")
    if os.path.exists(ref_so):
        theirs = subprocess.run(["nm", "-D", "--defined-only", ref_so], capture_output=True, text=True).stdout
        for name in want:
            ms = {l.split()[-1] for l in theirs.splitlines() if name in l}
            mo = {l.split()[-1] for l in ours.splitlines() if name in l}
            assert ms and ms == mo, (name, ms, mo)
    else:
        for name in want:
            assert name in ours
