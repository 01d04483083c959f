"""Parity of the CUDA substep with the oracle, through the C ABI (GPU tests).

The library evaluates a fixed sequence of IEEE operations per particle
(pbf_b200/csrc/pbf_device.cuh) and the oracle in product arithmetic evaluates
the same sequence on the CPU, so every field is compared bit for bit: cell
keys, cell starts, sorted order, neighbour lists, lambda, rho, dp, positions,
velocities, vorticity and XSPH terms, over one and several substeps.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pbf_b200 import Solver, scenes
from pbf_b200._lib import PBF_ERR_INVALID, PBF_ERR_NONFINITE, PBFError

from helpers import bits_equal, mismatch, oracle_original

pytestmark = pytest.mark.gpu


def make_pair(sc, debug=1, **ext):
    e = sc.ext(debug=debug, **ext)
    s = Solver(sc.para, sc.grid_space, sc.boundary, e)
    s.upload(sc.pos, sc.vel)
    orc = O.Oracle(O.params_for_scene(sc, ext), sc.pos, sc.vel)
    return s, orc


def assert_state_bitexact(s, orc, fields=("x", "v")):
    assert np.array_equal(s.fetch("perm"), orc.get("perm")), "perm"
    for name in fields:
        got = s.fetch(name)[:, :3]
        want = orc.get(name)
        n, d = mismatch(got, want)
        assert n == 0, f"{name}: {n} values differ (max abs {d})"


def assert_substep_bitexact(s, orc):
    """All intermediates of the last substep, in slot order."""
    assert np.array_equal(s.fetch("cell"), np.where(orc.get("cell") < 0, s.ncells, orc.get("cell"))), "cell"
    cs = s.fetch("cell_start")
    assert np.array_equal(cs[: s.ncells], orc.get("start")), "cell_start"
    assert np.array_equal(cs[1 : s.ncells + 1], orc.get("end")), "cell_end"
    assert cs[-1] == s.n
    assert np.array_equal(s.fetch("perm"), orc.get("perm")), "perm"
    assert np.array_equal(s.fetch("ncnt"), orc.get("ncnt")), "ncnt"
    nbr = s.fetch("nbr").reshape(s.max_neighbors, s.stride)[:, : s.n].T
    onb = orc.get("nbr").reshape(s.n, -1)
    cnt = orc.get("ncnt")
    mask = np.arange(s.max_neighbors)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, nbr, -1), onb), "nbr"
    for name, want in (("xpred", orc.get("xpred")), ("xold", orc.get("xold")), ("dp", orc.get("dp")),
                       ("curl", orc.get("curl")), ("vort", orc.get("vort")), ("visc", orc.get("visc")),
                       ("x", orc.get("x")), ("v", orc.get("v"))):
        n, d = mismatch(s.fetch(name)[:, :3], want)
        assert n == 0, f"{name}: {n} values differ (max abs {d})"
    assert bits_equal(s.fetch("xl")[:, 3], orc.get("lambda")), "lambda"
    assert bits_equal(s.fetch("rho"), orc.get("rho")), "rho"


@pytest.mark.parametrize("block,iters", [(16, 1), (16, 4), (32, 4)])
def test_single_substep_bitexact(block, iters):
    sc = scenes.dam_break(block, (40, 20, 20), stable=True, iterations=iters)
    s, orc = make_pair(sc)
    s.step(1)
    orc.substep()
    assert_substep_bitexact(s, orc)


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
@pytest.mark.parametrize("cell_scale", [1.0, 0.5])
def test_pair_lanes_bitexact(lanes, cell_scale):
    """Every pair-lane count: the neighbour lists are the single-thread lists and
    the lane sums follow the oracle's butterfly order bit for bit."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    ext = {"pair_lanes": lanes, "cell_scale": cell_scale,
           "grid_dims": [int(round(d / cell_scale)) for d in sc.ext_overrides["grid_dims"]]}
    s, orc = make_pair(sc, **ext)
    s.step(2)
    orc.substep(2)
    assert_substep_bitexact(s, orc)


def test_reference_formulas_single_substep_bitexact():
    """Reference parameter values without the stable-mode departures (the
    reference formulas, which diverge within a few substeps at these values)."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=False, iterations=4)
    s, orc = make_pair(sc)
    s.step(1)
    orc.substep()
    assert_substep_bitexact(s, orc)


def test_multi_substep_bitexact():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=4)
    s, orc = make_pair(sc, debug=0)
    for _ in range(3):
        s.step(4)
        orc.substep(4)
        assert_state_bitexact(s, orc)


def test_walls_outside_grid_descending_order_bitexact():
    """Fast particles in every direction (wall clamp with hashed offsets), a
    grid smaller than the box (out-of-grid bin), and the reference CPU's
    descending in-cell order."""
    sc = scenes.dam_break(12, (20, 10, 10), stable=False, iterations=2, grid_dims=(16, 8, 12))
    rng = np.random.RandomState(11)
    sc.vel = rng.uniform(-40, 40, size=sc.pos.shape).astype(np.float32)
    s, orc = make_pair(sc, cell_order=1)
    s.step(1)
    orc.substep()
    assert np.count_nonzero(orc.get("cell") < 0) > 0
    assert_substep_bitexact(s, orc)
    s.step(2)
    orc.substep(2)
    assert_state_bitexact(s, orc)


def test_neighbour_cap_binds_bitexact():
    """A compressed cloud where most particles have more than 63 neighbours
    (the cap of include/solverBase.h:6 must cut the list in stencil order)."""
    rng = np.random.RandomState(2)
    n = 3000
    pos = rng.uniform(0.5, 0.8, size=(n, 3)).astype(np.float32)
    sc = scenes.dam_break(4, (40, 20, 20), stable=True, iterations=2)
    sc.pos, sc.vel = pos, np.zeros_like(pos)
    sc.para.nParticles = n
    s, orc = make_pair(sc)
    s.step(1)
    orc.substep()
    assert (orc.get("ncnt") == 63).mean() > 0.5
    assert_substep_bitexact(s, orc)


@pytest.mark.parametrize("n", [1, 2, 33, 1000])
def test_small_and_ragged_counts(n):
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    sc.pos, sc.vel = sc.pos[:n].copy(), sc.vel[:n].copy()
    sc.para.nParticles = n
    s, orc = make_pair(sc)
    s.step(2)
    orc.substep(2)
    assert_substep_bitexact(s, orc)


def test_sphere_obstacle_bitexact():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    sph = (0.45, 0.25, 0.45, 0.2)
    s, orc = make_pair(sc, sphere=sph)
    s.step(3)
    orc.substep(3)
    assert_state_bitexact(s, orc)
    x = s.fetch("x")[:, :3]
    d = np.linalg.norm(x - np.float32(sph[:3]), axis=1)
    assert d.min() >= sph[3] * (1 - 1e-5)


def test_grid_build_vs_reference_cpu_buildNeiborhood():
    """Hash, counts, scan, cell ranges and sorted order bit-exact against the
    reference CPU solver's buildNeiborhood on the same positions (descending
    in-cell order, the reference CPU's); neighbour sets equal."""
    if not O.refcpu_available():
        pytest.skip("reference CPU solver not built here")
    sc = scenes.dam_break(16, (40, 20, 20), stable=False)
    rng = np.random.RandomState(4)
    pos = (sc.pos + rng.uniform(-0.02, 0.02, sc.pos.shape)).astype(np.float32)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(grid_dims=[64, 64, 64], cell_order=1, debug=1))
    s.upload(pos, sc.vel)
    s.build_grid()
    ref = O.RefCpu(sc.para, sc.grid_space)
    ref.build(pos)
    hash_ = s.fetch("hash")
    rc = ref.get("cell")
    assert np.array_equal(np.where(hash_ == s.ncells, -1, hash_), rc)
    cs = s.fetch("cell_start")
    assert np.array_equal(cs[: s.ncells], ref.get("start"))
    assert np.array_equal(cs[1 : s.ncells + 1], ref.get("end"))
    inside = int(np.count_nonzero(rc >= 0))
    assert np.array_equal(s.fetch("perm")[:inside], ref.get("sorted")[:inside])
    perm = s.fetch("perm")
    lists = s.neighbor_lists()
    rn = ref.get("nbr").reshape(s.n, 63)
    rcnt = ref.get("ncnt")
    for k in range(s.n):
        i = perm[k]
        got = sorted(int(perm[j]) for j in lists[k])
        want = sorted(int(x) for x in rn[i, : rcnt[i]])
        assert got == want, k


@pytest.mark.parametrize("m", [1, 31, 2047, 2048, 2049, 4095, 4096, 4097, 64 ** 3, 1_000_003, 1 << 21, (1 << 21) + 1,
                               (1 << 22) - 1, 1 << 22, 8_192_001])
def test_scan_matches_exclusive_prefix(m):
    """pbf_scan_exclusive_i32 on the shape of test/testPrefixSum.cpp:65-85
    (values rand()%16) and on ragged / large sizes; the total lands at out[m]."""
    import torch
    from pbf_b200._lib import lib, check
    rng = np.random.RandomState(m % 1000)
    a = rng.randint(0, 16, size=m).astype(np.int32)
    d_in = torch.from_numpy(a).cuda()
    d_out = torch.empty(m + 1, dtype=torch.int32, device="cuda")
    ws_bytes = lib().pbf_scan_workspace_bytes(m)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    check(lib().pbf_scan_exclusive_i32(d_in.data_ptr(), d_out.data_ptr(), m, ws.data_ptr(), ws_bytes, None))
    want = np.concatenate([[0], np.cumsum(a, dtype=np.int64)]).astype(np.int32)
    assert np.array_equal(d_out.cpu().numpy(), want)
    assert np.array_equal(d_in.cpu().numpy(), a), "input must be left unchanged"


@pytest.mark.parametrize("m", [1, 4099, 262144 + 3, (1 << 22) + 3])
@pytest.mark.parametrize("shift", [1, 3])
def test_scan_unaligned_pointers(m, shift):
    """Arrays that do not start on a 16-byte boundary take the scalar path of the
    scan (aligned ones move four counts per access); both give the same prefix."""
    import torch
    from pbf_b200._lib import lib, check
    rng = np.random.RandomState(m + shift)
    a = rng.randint(0, 16, size=m).astype(np.int32)
    buf_in = torch.zeros(m + 8, dtype=torch.int32, device="cuda")
    buf_in[shift:shift + m] = torch.from_numpy(a).cuda()
    buf_out = torch.full((m + 8,), -7, dtype=torch.int32, device="cuda")
    ws_bytes = lib().pbf_scan_workspace_bytes(m)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    check(lib().pbf_scan_exclusive_i32(buf_in[shift:].data_ptr(), buf_out[shift:].data_ptr(), m, ws.data_ptr(),
                                       ws_bytes, None))
    want = np.concatenate([[0], np.cumsum(a, dtype=np.int64)]).astype(np.int32)
    out = buf_out.cpu().numpy()
    assert np.array_equal(out[shift:shift + m + 1], want)
    assert np.all(out[:shift] == -7) and np.all(out[shift + m + 1:] == -7)


def test_density_error_vs_fp64_oracle():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=4)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(measure_error=1))
    s.upload(sc.pos, sc.vel)
    s.step(5)
    st = s.stats()
    pos, _ = s.download()
    mx, mean = O.density_error(pos, float(sc.para.h), float(sc.para.restRho))
    assert abs(st["max_density_error"] - mx) <= 1e-4
    assert abs(st["mean_density_error"] - mean) <= 1e-5


def test_adaptive_iterations_reach_tolerance():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=1)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(adaptive=1, density_tol=0.005, max_iterations=12))
    s.upload(sc.pos, sc.vel)
    total = 0
    for k in range(4):
        s.step(1)
        st = s.stats()
        assert st["max_density_error"] <= 0.005 or st["last_iterations"] == 12
        assert 1 <= st["last_iterations"] <= 12
        total += st["last_iterations"]
        assert st["substeps"] == k + 1 and st["total_iterations"] == total
    pos, _ = s.download()
    mx, _ = O.density_error(pos, float(sc.para.h), float(sc.para.restRho))
    assert mx <= 0.005 + 1e-4 or st["last_iterations"] == 12


@pytest.mark.parametrize("profile", [0, 1])
def test_adaptive_loop_bitexact(profile):
    """The adaptive corrections (a device-side graph while loop; unrolled when
    profiling) against the oracle's adaptive substep: the same correction count
    every substep and bit-identical state."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=1)
    s, orc = make_pair(sc, adaptive=1, density_tol=0.005, max_iterations=12, profile=profile)
    tol = float(np.float32(0.005))
    counts = []
    for _ in range(4):
        s.step(1)
        want = orc.substep_adaptive(tol, 1, 12)
        counts.append(want)
        assert s.stats()["last_iterations"] == want
        assert_state_bitexact(s, orc)
    assert max(counts) > 1  # the tolerance made the loop run more than once
    plain = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(adaptive=1, density_tol=0.005, max_iterations=12,
                                                               profile=1 - profile))
    if profile == 0:  # one pass of the loop body counts once
        assert s.kernel_count() < plain.kernel_count()


def test_build_grid_between_substeps_bitexact():
    """A grid build between substeps re-sorts the state and sets up the next
    substep's grid hash (which the vorticity pass otherwise provides): the
    following substeps still match the oracle bit for bit."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    s, orc = make_pair(sc, debug=0)
    s.step(2)
    orc.substep(2)
    s.build_grid()
    orc.build_only()
    assert_state_bitexact(s, orc)
    s.step(2)
    orc.substep(2)
    assert_state_bitexact(s, orc)
    # and an upload of the current state in the middle of a run
    pos, vel = s.download()
    s.upload(pos, vel)
    orc2 = O.Oracle(O.params_for_scene(sc), pos, vel)
    s.step(2)
    orc2.substep(2)
    assert_state_bitexact(s, orc2)


def test_host_errors():
    sc = scenes.dam_break(4, (40, 20, 20))
    with pytest.raises(PBFError) as e:
        Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(max_neighbors=0))
    assert e.value.code == PBF_ERR_INVALID
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    bad = sc.pos.copy()
    bad[3, 1] = np.nan
    with pytest.raises(PBFError) as e:
        s.upload(bad, sc.vel)
    assert e.value.code == PBF_ERR_NONFINITE
    with pytest.raises(PBFError):
        s.step(1)  # nothing uploaded


def test_drop_in_entry_points_and_bound_position():
    """initCUDASolverDataBuffer / cudaPBFSolve / freeCUDASolverDataBuffer, with
    a caller-owned device position buffer refreshed in original order after
    every substep (the reference app's mapped VBO)."""
    import torch
    import pbf_b200 as P
    sc = scenes.dam_break(16, (40, 20, 20), stable=True)
    data = P.initCUDASolverDataBuffer(sc.pos, sc.vel, sc.para, sc.grid_space, sc.boundary, sc.ext())
    buf = torch.zeros((sc.n, 3), dtype=torch.float32, device="cuda")
    data.bind_position(buf)
    orc = O.Oracle(O.params_for_scene(sc), sc.pos, sc.vel)
    for _ in range(3):
        P.cudaPBFSolve(data, sc.para)
        orc.substep()
        torch.cuda.synchronize()
        assert bits_equal(buf.cpu().numpy(), oracle_original(orc, "x").astype(np.float32))
    P.freeCUDASolverDataBuffer(data)


def test_step_host_pipelined_frames():
    """pbf_step_host: every call uploads its own host inputs, runs a substep and
    copies the positions back; with double-buffered staging, interleaved calls on
    two different states each give the positions of a plain upload, step and
    download of that state."""
    import torch
    sc = scenes.dam_break(16, (40, 20, 20), stable=True)
    a = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    b = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    b.upload(sc.pos, sc.vel)
    b.step(3)
    pos2, vel2 = b.download()
    want = []
    for pos, vel in ((sc.pos, sc.vel), (pos2, vel2)):
        b.upload(pos, vel)
        b.step(1)
        want.append(b.download()[0])
    ins = [(torch.from_numpy(np.ascontiguousarray(p, np.float32)).pin_memory(),
            torch.from_numpy(np.ascontiguousarray(v, np.float32)).pin_memory()) for p, v in ((sc.pos, sc.vel), (pos2, vel2))]
    outs = [torch.empty((sc.n, 3), dtype=torch.float32).pin_memory() for _ in range(4)]
    stream = torch.cuda.Stream()
    for k in range(4):
        a.step_host(ins[k % 2][0], ins[k % 2][1], outs[k], 1, stream)
    a.host_fence(stream)
    stream.synchronize()
    for k in range(4):
        assert bits_equal(outs[k].numpy(), want[k % 2]), k


@pytest.mark.parametrize("fail_at", [1, 2, 4])
def test_step_host_staging_failure_leaves_the_handle_retryable(fail_at):
    """A staging allocation of pbf_step_host that fails (injected on the host)
    returns PBF_ERR_ALLOC and attaches nothing; the next call sets the staging
    up again and gives the positions of a plain upload, step and download."""
    import torch
    from pbf_b200._lib import PBF_ERR_ALLOC, check, lib
    sc = scenes.dam_break(12, (40, 20, 20), stable=True)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    ref = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    ref.upload(sc.pos, sc.vel)
    ref.step(1)
    want = ref.download()[0]
    pos = torch.from_numpy(np.ascontiguousarray(sc.pos, np.float32)).pin_memory()
    vel = torch.from_numpy(np.ascontiguousarray(sc.vel, np.float32)).pin_memory()
    out = torch.zeros((sc.n, 3), dtype=torch.float32).pin_memory()
    stream = torch.cuda.Stream()
    check(lib().pbf_debug_fail_staging_alloc(fail_at))
    try:
        with pytest.raises(PBFError) as e:
            s.step_host(pos, vel, out, 1, stream)
        assert e.value.code == PBF_ERR_ALLOC
    finally:
        check(lib().pbf_debug_fail_staging_alloc(0))
    s.step_host(pos, vel, out, 1, stream)
    s.host_fence(stream)
    stream.synchronize()
    assert bits_equal(out.numpy(), want)
    s.close()
    ref.close()
