"""The allocation-free scan (GPU test, collected last on purpose).

pbf_scan_exclusive_i32_noalloc serves callers that cannot call cudaMalloc (a
frame loop that must not stall, a plug-in whose host owns all device memory):
its scratch lives in a device array inside the library. It must give exactly
what the workspace-taking pbf_scan_exclusive_i32 gives, on consecutive calls
that reuse the shared array, and refuse sizes beyond its stated maximum.
"""
import numpy as np
import pytest
import torch

from pbf_b200._lib import PBF_ERR_INVALID, check, lib

pytestmark = pytest.mark.gpu

MAX_N = 16_777_216


def scan_with_workspace(d_in, n):
    out = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    ws_bytes = lib().pbf_scan_workspace_bytes(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    check(lib().pbf_scan_exclusive_i32(d_in.data_ptr(), out.data_ptr(), n, ws.data_ptr(), ws_bytes, None))
    return out


def scan_no_alloc(d_in, n):
    out = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    check(lib().pbf_scan_exclusive_i32_noalloc(d_in.data_ptr(), out.data_ptr(), n, None))
    return out


def test_no_alloc_scan_matches_the_workspace_scan_on_consecutive_calls():
    rng = np.random.RandomState(123)
    # two calls in a row: the second reuses (and must clear) the shared scratch
    for n in (1_000_003, 262_145):
        a = torch.from_numpy(rng.randint(0, 16, size=n).astype(np.int32)).cuda()
        want = scan_with_workspace(a, n)
        got = scan_no_alloc(a, n)
        torch.cuda.synchronize()
        assert torch.equal(got, want), n
        assert int(got[-1]) == int(a.sum())


def test_no_alloc_scan_limits():
    a = torch.ones(MAX_N, dtype=torch.int32, device="cuda")
    got = scan_no_alloc(a, MAX_N)
    assert int(got[-1]) == MAX_N and int(got[12345]) == 12345
    out = torch.empty(8, dtype=torch.int32, device="cuda")
    assert lib().pbf_scan_exclusive_i32_noalloc(a.data_ptr(), out.data_ptr(), MAX_N + 1, None) == PBF_ERR_INVALID
    assert b"16,777,216" in lib().pbf_last_error()
