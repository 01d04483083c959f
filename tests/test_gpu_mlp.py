"""Learned lambda warm start (GPU tests).

* the tensor-core forward pass and gradients against the CPU FP64 oracle of the
  same network (oracle/mlp_oracle.py);
* training on the GPU reduces the loss;
* recording features changes no solver result, and the features match a CPU
  recomputation from the solver's own state;
* end to end: a network trained on trajectories this solver generates lowers
  the density error of a 2-iteration substep compared with 2 plain iterations.
"""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M
from oracle import oracle as O
from pbf_b200 import Solver, learned, scenes

pytestmark = pytest.mark.gpu


def random_params(seed, feat, target):
    w, b = learned.init_params(seed)
    b = learned.set_normalisation(b, feat, target)
    rng = np.random.RandomState(seed)
    b[:193] = rng.normal(0, 0.1, 193).astype(np.float32)  # non-zero biases exercise their gradients
    return w, b


def random_rows(n, seed):
    rng = np.random.RandomState(seed)
    scales = np.float32([0.5, 1.1, 2e-5, 300.0, 3.0, 2.0, 2.0, 2.0, 8.0, 8.0, 0.7, 15.0])
    feat = (rng.normal(0, 1, (n, 12)) * scales + scales).astype(np.float32)
    target = (np.tanh(feat[:, 1] - 1.0) * 3e-5 + 1e-6 * feat[:, 4]).astype(np.float32)
    return feat, target


def test_forward_matches_fp64_oracle():
    feat, target = random_rows(1000, 1)
    w, b = random_params(1, feat, target)
    tr = learned.Trainer(w, b, max_batch=1024)
    got = tr.forward(torch.from_numpy(feat).cuda()).cpu().numpy().astype(np.float64)
    want, _ = M.forward(w, b, feat)
    scale = np.sqrt(np.mean(want ** 2))
    assert np.abs(got - want).max() <= 2e-2 * scale, np.abs(got - want).max() / scale
    tr.close()


@pytest.mark.parametrize("n", [128, 600, 4096])
def test_gradients_match_fp64_oracle(n):
    feat, target = random_rows(n, 2)
    w, b = random_params(2, feat, target)
    tr = learned.Trainer(w, b, max_batch=4096)
    gw, gb, loss = tr.gradients(torch.from_numpy(feat).cuda(), torch.from_numpy(target).cuda())
    rw, rb, rloss = M.gradients(w, b, feat, target)
    assert abs(loss - rloss) <= 2e-2 * rloss
    blocks = [("W1", gw[M.W1:M.W2], rw[M.W1:M.W2]), ("W2", gw[M.W2:M.W3], rw[M.W2:M.W3]),
              ("W3", gw[M.W3:M.W4], rw[M.W3:M.W4]), ("w4", gw[M.W4:], rw[M.W4:]),
              ("b1", gb[0:64], rb[0:64]), ("b2", gb[64:128], rb[64:128]), ("b3", gb[128:192], rb[128:192]),
              ("b4", gb[192:193], rb[192:193])]
    for name, g, r in blocks:
        rel = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)
        cos = float(np.dot(g, r) / max(np.linalg.norm(g) * np.linalg.norm(r), 1e-30))
        assert rel <= 4e-2 and cos >= 0.999, (name, rel, cos)
    assert np.all(gb[193:] == 0)  # normalisation constants are not trained
    tr.close()


def test_training_reduces_loss():
    feat, target = random_rows(16384, 3)
    ft, tt = torch.from_numpy(feat).cuda(), torch.from_numpy(target).cuda()
    tr, losses = learned.train(ft, tt, epochs=20, batch=2048, lr=3e-3, log_every=1)
    first, last = losses[0][1], losses[-1][1]
    assert last < 0.1 * first, (first, last)
    tr.close()


def test_training_is_reproducible():
    """The gradients are summed per tile and warp and then in a fixed order (no
    floating-point atomics), so the same rows and seed give the same weights bit
    for bit, and the same warm-started solver state after them."""
    feat, target = random_rows(8192 + 300, 5)  # a partial last tile
    ft, tt = torch.from_numpy(feat).cuda(), torch.from_numpy(target).cuda()
    out = []
    for _ in range(2):
        tr, losses = learned.train(ft, tt, epochs=2, batch=2048, lr=3e-3, log_every=1)
        w32, b32, w16 = tr.params()
        tr.close()
        out.append((w32, b32, w16, [l for _, l in losses]))
    w_a, b_a, h_a, l_a = out[0]
    w_b, b_b, h_b, l_b = out[1]
    assert np.array_equal(w_a.view(np.uint32), w_b.view(np.uint32))
    assert np.array_equal(b_a.view(np.uint32), b_b.view(np.uint32))
    assert np.array_equal(h_a, h_b)
    assert l_a == l_b


def test_recording_features_changes_nothing():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=3)
    a = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext())
    b = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(record_features=1))
    for s in (a, b):
        s.upload(sc.pos, sc.vel)
        s.step(4)
    for name in ("x", "v", "perm"):
        assert np.array_equal(a.fetch(name).view(np.uint32), b.fetch(name).view(np.uint32)), name


def test_features_match_cpu_recomputation():
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=2)
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(record_features=1, debug=1))
    s.upload(sc.pos, sc.vel)
    s.step(1)
    lam1, perm1 = s.fetch("lambda_total"), s.fetch("perm")
    s.step(1)
    f = s.fetch("features")
    perm2 = s.fetch("perm")
    xp = s.fetch("xpred")[:, :3].astype(np.float64)
    ncnt = s.fetch("ncnt")
    nbr = s.fetch("nbr").reshape(s.max_neighbors, s.stride)
    h, rho0 = float(sc.para.h), float(sc.para.restRho)
    assert np.allclose(f[:, 0], ncnt / 63.0, rtol=0, atol=1e-7)
    # previous substep's total lambda, carried through the re-sort
    slot_of = np.empty(s.n, np.int64)
    slot_of[perm1] = np.arange(s.n)
    assert np.array_equal(f[:, 2], lam1[slot_of[perm2]])
    # fluid density from the same neighbour lists
    c6 = 315.0 / (64.0 * np.pi * h ** 9)
    rho = np.zeros(s.n)
    for q in range(s.max_neighbors):
        m = ncnt > q
        if not m.any():
            break
        j = nbr[q, : s.n][m]
        r2 = ((xp[m] - xp[j]) ** 2).sum(1)
        rho[m] += np.where(r2 <= h * h, c6 * np.maximum(h * h - r2, 0) ** 3, 0.0)
    assert np.allclose(f[:, 1], rho / rho0, rtol=2e-5, atol=1e-6)
    # wall distances
    lo, hi = np.array(sc.boundary[:3]), np.array(sc.boundary[3:])
    dw = np.clip(np.minimum(xp - lo, hi - xp) / h, 0, 4)
    assert np.allclose(f[:, 5:8], dw, atol=1e-5)
    # close neighbours, neighbourhood offset and |sum grad W| from the same lists
    close = np.zeros(s.n)
    roff = np.zeros((s.n, 3))
    gsum = np.zeros((s.n, 3))
    spiky = -45.0 / (np.pi * h ** 6)
    for q in range(s.max_neighbors):
        m = ncnt > q
        if not m.any():
            break
        j = nbr[q, : s.n][m]
        r = xp[m] - xp[j]
        r2 = (r ** 2).sum(1)
        close[m] += r2 < 0.25 * h * h
        roff[m] += r
        rl = np.sqrt(r2)
        ok = (rl <= h) & (rl >= 0.01)
        coef = np.where(ok, spiky * (h - rl) ** 2 / np.maximum(rl, 1e-30), 0.0)
        gsum[m] += coef[:, None] * r
    assert np.array_equal(f[:, 8], (close / 63.0).astype(np.float32))
    cnt1 = np.maximum(ncnt, 1)
    assert np.allclose(f[:, 9], np.linalg.norm(roff, axis=1) / (h * cnt1), rtol=1e-4, atol=1e-5)
    assert np.allclose(f[:, 10], np.linalg.norm(gsum, axis=1) * h / rho0, rtol=1e-3, atol=1e-4)
    assert np.all(np.isfinite(f[:, 11])) and np.all(f[:, 11] >= 0)


def _run_errors(sc, ext, steps, w16=None, b32=None):
    s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(measure_error=1, **ext))
    if w16 is not None:
        learned.install(s, w16, b32)
    s.upload(sc.pos, sc.vel)
    mx, mean = [], []
    for _ in range(steps):
        s.step(1)
        st = s.stats()
        mx.append(st["max_density_error"])
        mean.append(st["mean_density_error"])
    s.close()
    return float(np.mean(mx)), float(np.mean(mean))


def test_warm_start_beats_the_same_iterations_without_it():
    """Trained on 160 substeps of this solver's own 4-iteration trajectory, the
    network makes a 2-iteration substep (lambda0 + 1 plain iteration) more
    accurate than 2 plain iterations, over the same scene."""
    sc4 = scenes.dam_break(24, (40, 20, 20), stable=True, iterations=4)
    feat, target = learned.collect(sc4, substeps=160, rows_per_substep=4096, seed=0)
    tr, losses = learned.train(feat, target, epochs=4, batch=4096, lr=2e-3, log_every=50)
    w, b, w16 = tr.params()
    tr.close()
    sc2 = scenes.dam_break(24, (40, 20, 20), stable=True, iterations=2)
    plain2 = _run_errors(sc2, {}, 80)
    warm2 = _run_errors(sc2, {"warm_start": 1}, 80, w16, b)
    print(f"losses {losses[0][1]:.4g} -> {losses[-1][1]:.4g}; mean density error: plain x2 {plain2[1]:.5f}, "
          f"warm+1 {warm2[1]:.5f}; max: {plain2[0]:.4f} vs {warm2[0]:.4f}")
    assert warm2[1] < plain2[1]


def test_collect_batch_rows():
    """Training rows gathered from a batch of scenes: finite features, the
    neighbour fraction in [0, 1], and a non-trivial total lambda."""
    scs = scenes.config2(seed=3, n_scenes=3, lo=300, hi=1500, iterations=3)
    feat, target = learned.collect_batch(scs, substeps=4, rows_per_substep=64, seed=1)
    f, t = feat.cpu().numpy(), target.cpu().numpy()
    assert f.shape == (256, 12) and t.shape == (256,)
    assert np.isfinite(f).all() and np.isfinite(t).all()
    assert (f[:, 0] >= 0).all() and (f[:, 0] <= 1).all()
    assert np.abs(t).max() > 0


@pytest.mark.parametrize("lanes,block,persistent,clamp,floor", [(2, 256, 0, 4.0, 0), (2, 256, 1, 0.0, 0),
                                                                (1, 128, 0, 4.0, 1), (4, 256, 0, 0.0, 0),
                                                                (2, 64, 1, 4.0, 1), (1, 256, 0, 16.0, 1)])
def test_fused_warm_pass_matches_the_two_launch_path(lanes, block, persistent, clamp, floor):
    """The fused first pass (features on chip, the network on the tensor cores in
    the same kernel) gives the two-launch path's lambda0, total lambda and state
    bit for bit over several substeps, for every tile shape (256, 128, 64 or 32
    rows per block: two, one or a partial MMA tile)."""
    sc = scenes.dam_break(20, (40, 20, 20), stable=True, iterations=2)
    feat, target = learned.collect(sc, substeps=30, rows_per_substep=2048, seed=0)
    tr, _ = learned.train(feat, target, epochs=1, batch=2048, lr=2e-3)
    _, b32, w16 = tr.params()
    tr.close()
    ext = dict(warm_start=1, pair_lanes=lanes, block_size=block, persistent=persistent, warm_clamp=clamp,
               warm_floor=floor, record_features=1)
    runs = []
    for unfused in (0, 1):
        s = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(warm_unfused=unfused, **ext))
        learned.install(s, w16, b32)
        s.upload(sc.pos, sc.vel)
        s.step(4)
        assert s.stats()["error_bits"] == 0
        runs.append({k: s.fetch(k) for k in ("lambda0", "lambda_total", "x", "v", "features")})
        s.close()
    for k in runs[0]:
        assert np.array_equal(runs[0][k].view(np.uint32), runs[1][k].view(np.uint32)), k
    assert np.abs(runs[0]["lambda0"]).max() > 0


def test_trust_region_floor_keeps_lambda0_between_the_plain_lambda_and_its_multiple():
    """With warm_floor, lambda0 lies between the plain lambda of its pass and
    warm_clamp times it: the first correction never pushes less than a plain
    iteration would. The plain lambda is that of a solver without the warm start
    stepped once from the same upload (one correction: its total lambda)."""
    sc = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=2)
    feat, target = learned.collect(sc, substeps=20, rows_per_substep=1024, seed=0)
    tr, _ = learned.train(feat, target, epochs=1, batch=1024, lr=2e-3)
    _, b32, w16 = tr.params()
    tr.close()
    sc1 = scenes.dam_break(16, (40, 20, 20), stable=True, iterations=1)
    warm = Solver(sc1.para, sc1.grid_space, sc1.boundary, sc1.ext(warm_start=1, warm_clamp=3.0, warm_floor=1))
    learned.install(warm, w16, b32)
    plain = Solver(sc1.para, sc1.grid_space, sc1.boundary, sc1.ext(record_features=1))
    for s in (warm, plain):
        s.upload(sc1.pos, sc1.vel)
        s.step(1)
    l0 = warm.fetch("lambda0")
    lp = plain.fetch("lambda_total")
    assert np.array_equal(warm.fetch("perm"), plain.fetch("perm"))
    lo = np.minimum(lp, np.float32(3.0) * lp)
    hi = np.maximum(lp, np.float32(3.0) * lp)
    assert np.all(l0 >= lo) and np.all(l0 <= hi)
    assert np.count_nonzero(lp) > 0 and np.count_nonzero(l0 != lp) > 0
    warm.close()
    plain.close()
