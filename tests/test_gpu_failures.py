"""Failure detection on the device without a GPU fault (GPU tests).

The reference stops the process on any CUDA error (CHECK_CUDA,
kernels/cudaPBFSolver.cuh:5-10). Here every spin-wait in a kernel is bounded:
the scan's decoupled look-back (waiting for a predecessor tile's status) and
the warm-start network's waits on its tensor-core barrier. When a wait runs out
the kernel records PBF_DEVERR_* in the handle's error word, frees what it holds
and returns, and the host reports PBF_ERR_DEVICE. pbf_debug_expire_wait runs the
production kernels with a wait that nothing will satisfy (a tile that never
publishes, a barrier nothing is committed to) and a short limit; these tests
check the status that comes back and that the context keeps working.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import Solver, scenes
from pbf_b200._lib import PBF_DEVERR_MLP_TIMEOUT, PBF_DEVERR_SCAN_TIMEOUT, PBF_ERR_DEVICE, lib

pytestmark = pytest.mark.gpu


def scan_still_correct():
    import torch
    from pbf_b200._lib import check
    m = 100_003
    a = np.random.RandomState(1).randint(0, 16, size=m).astype(np.int32)
    d_in = torch.from_numpy(a).cuda()
    d_out = torch.empty(m + 1, dtype=torch.int32, device="cuda")
    ws_bytes = lib().pbf_scan_workspace_bytes(m)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    check(lib().pbf_scan_exclusive_i32(d_in.data_ptr(), d_out.data_ptr(), m, ws.data_ptr(), ws_bytes, None))
    want = np.concatenate([[0], np.cumsum(a, dtype=np.int64)]).astype(np.int32)
    return np.array_equal(d_out.cpu().numpy(), want)


def substep_still_bitexact():
    sc = scenes.dam_break(8, (40, 20, 20), stable=True, iterations=2)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    s.upload(sc.pos, sc.vel)
    s.step(2)
    assert s.stats()["error_bits"] == 0
    orc = O.Oracle(O.params_for_scene(sc), sc.pos, sc.vel)
    orc.substep(2)
    x = s.fetch("x")[:, :3]
    return np.array_equal(x.view(np.uint32), orc.get("x").astype(np.float32).view(np.uint32))


@pytest.mark.parametrize("which,bit", [(0, PBF_DEVERR_SCAN_TIMEOUT), (1, PBF_DEVERR_MLP_TIMEOUT)])
def test_expired_wait_is_reported_and_the_context_stays_usable(which, bit):
    bits = C.c_int(-1)
    rc = lib().pbf_debug_expire_wait(which, C.byref(bits))
    assert rc == PBF_ERR_DEVICE, lib().pbf_last_error()
    assert bits.value == bit
    assert b"error bits" in lib().pbf_last_error()
    assert scan_still_correct()
    assert substep_still_bitexact()

