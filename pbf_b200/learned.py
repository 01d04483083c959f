"""Learned lambda warm start: collect training rows from the solver, train the
per-particle MLP on the GPU with the library's tensor-core forward/backward
kernels, and install it into a solver.

The target of a row is the total lambda the plain Jacobi loop applied to that
particle in its substep (the sum over iterations); the 12 features come from the
first lambda pass of the same substep (see pbf_kernels.cu: k_features). Applied
as the first correction, the prediction stands in for several plain iterations.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, lib

NUM_W = _lib.MLP_NUM_WEIGHTS
NUM_B = _lib.MLP_NUM_BIASES
W1, W2, W3, W4 = 0, 64 * 16, 64 * 16 + 64 * 64, 64 * 16 + 2 * 64 * 64
B1, B2, B3, B4, FMEAN, FISTD, OSCALE = 0, 64, 128, 192, 193, 209, 225
FEATURES = ["neighbour_fraction", "density", "previous_total_lambda", "grad_c_sq", "divergence", "wall_x",
            "wall_y", "wall_z", "close_fraction", "neighbourhood_offset", "grad_w_sum", "velocity_spread"]


def init_params(seed: int = 0):
    """Glorot-uniform weights (the 4 padding inputs of layer 1 zero), zero
    biases, identity normalisation, unit output scale."""
    rng = np.random.RandomState(seed)
    w = np.zeros(NUM_W, np.float32)

    def glorot(fan_in, fan_out, shape):
        a = np.sqrt(6.0 / (fan_in + fan_out))
        return rng.uniform(-a, a, size=shape).astype(np.float32)

    w1 = np.zeros((64, 16), np.float32)
    w1[:, :12] = glorot(12, 64, (64, 12))
    w[W1:W2] = w1.ravel()
    w[W2:W3] = glorot(64, 64, (64, 64)).ravel()
    w[W3:W4] = glorot(64, 64, (64, 64)).ravel()
    w[W4:] = glorot(64, 1, (64,)) * 0.5
    b = np.zeros(NUM_B, np.float32)
    b[FISTD:FISTD + 12] = 1.0
    b[OSCALE] = 1.0
    return w, b


def set_normalisation(b: np.ndarray, feat: np.ndarray, target: np.ndarray) -> np.ndarray:
    """Feature mean / (1/std) and the output scale (rms of the targets) from a dataset."""
    b = b.copy()
    f = np.asarray(feat, np.float64)
    mean = f.mean(0)
    std = f.std(0)
    b[FMEAN:FMEAN + 12] = mean.astype(np.float32)
    b[FISTD:FISTD + 12] = np.where(std > 1e-12, 1.0 / np.maximum(std, 1e-30), 0.0).astype(np.float32)
    rms = float(np.sqrt(np.mean(np.asarray(target, np.float64) ** 2)))
    b[OSCALE] = np.float32(rms if rms > 0 else 1.0)
    return b


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16 bit patterns."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


class Trainer:
    """pbf_mlp_trainer: FP32 masters, Adam state, tensor-core kernels."""

    def __init__(self, w32: np.ndarray, b32: np.ndarray, max_batch: int = 8192):
        self.max_batch = max_batch
        w = np.ascontiguousarray(w32, np.float32)
        b = np.ascontiguousarray(b32, np.float32)
        h = C.c_void_p()
        check(lib().pbf_mlp_trainer_create(max_batch, w.ctypes.data, b.ctypes.data, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pbf_mlp_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gradients(self, feat, target):
        """(grad of weights [9280], grad of biases [226], loss) for device tensors."""
        gw = np.zeros(NUM_W, np.float32)
        gb = np.zeros(NUM_B, np.float32)
        loss = np.zeros(1, np.float32)
        check(lib().pbf_mlp_gradients(self._h, feat.data_ptr(), target.data_ptr(), int(feat.shape[0]),
                                      gw.ctypes.data, gb.ctypes.data, loss.ctypes.data, None))
        return gw, gb, float(loss[0])

    def step(self, feat, target, lr: float, want_loss: bool = False):
        loss = np.zeros(1, np.float32)
        check(lib().pbf_mlp_train_step(self._h, feat.data_ptr(), target.data_ptr(), int(feat.shape[0]), float(lr),
                                       loss.ctypes.data if want_loss else None, None))
        return float(loss[0]) if want_loss else None

    def forward(self, feat):
        import torch
        out = torch.empty(feat.shape[0], dtype=torch.float32, device=feat.device)
        check(lib().pbf_mlp_forward(self._h, feat.data_ptr(), int(feat.shape[0]), out.data_ptr(), None))
        return out

    def params(self):
        w = np.zeros(NUM_W, np.float32)
        b = np.zeros(NUM_B, np.float32)
        w16 = np.zeros(NUM_W, np.uint16)
        check(lib().pbf_mlp_get_params(self._h, w.ctypes.data, b.ctypes.data, w16.ctypes.data))
        return w, b, w16


def install(solver, w16: np.ndarray, b32: np.ndarray) -> None:
    """Installs BF16 weights and constants into a solver (ext.warm_start must be set to use them)."""
    w = np.ascontiguousarray(w16, np.uint16)
    b = np.ascontiguousarray(b32, np.float32)
    check(lib().pbf_set_warm_start(solver.handle, w.ctypes.data, w.size, b.ctypes.data, b.size))


def collect(scene, substeps: int, rows_per_substep: int, seed: int = 0, warmup: int = 0, ext: Optional[dict] = None):
    """Runs the plain solver on `scene` and gathers `rows_per_substep` random
    particles' (features, total lambda) after every substep. Returns device
    tensors feat [S, 12], target [S]."""
    from .solver import Solver
    kw = dict(ext or {})
    kw["record_features"] = 1
    s = Solver(scene.para, scene.grid_space, scene.boundary, scene.ext(**kw))
    s.upload(scene.pos, scene.vel)
    if warmup:
        s.step(warmup)
    try:
        return collect_from(s, substeps, rows_per_substep, seed)
    finally:
        s.close()


def collect_batch(scenes_, substeps: int, rows_per_substep: int, seed: int = 0, ext: Optional[dict] = None):
    """collect() on a batch of scenes (pbf_b200.scenes.batch_inputs) run as one BatchSolver."""
    from . import scenes as S
    from .solver import BatchSolver
    para, descs, ov, pos, vel = S.batch_inputs(scenes_)
    ov.update(ext or {})
    ov["record_features"] = 1
    b = BatchSolver(para, descs, S.default_ext(**ov))
    b.upload(pos, vel)
    try:
        return collect_from(b, substeps, rows_per_substep, seed)
    finally:
        b.close()


def collect_from(s, substeps: int, rows_per_substep: int, seed: int = 0):
    """Steps an uploaded solver created with record_features = 1 and gathers
    `rows_per_substep` random particles' (features, total lambda) after every substep."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    total = substeps * rows_per_substep
    feat = torch.empty((total, 12), dtype=torch.float32, device="cuda")
    target = torch.empty(total, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    for t in range(substeps):
        s.step(1, stream)
        slots = torch.randint(0, s.n, (rows_per_substep,), generator=g, device="cuda", dtype=torch.int32)
        a, b = t * rows_per_substep, (t + 1) * rows_per_substep
        check(lib().pbf_gather_training_rows(s.handle, slots.data_ptr(), rows_per_substep, feat[a:b].data_ptr(),
                                             target[a:b].data_ptr(), int(stream.cuda_stream)))
    torch.cuda.synchronize()
    return feat, target


def train(feat, target, epochs: int = 4, batch: int = 4096, lr: float = 2e-3, seed: int = 0, log_every: int = 0):
    """Trains from Glorot initialisation with Adam; returns (Trainer, losses)."""
    import torch
    w, b = init_params(seed)
    b = set_normalisation(b, feat.cpu().numpy(), target.cpu().numpy())
    tr = Trainer(w, b, max_batch=batch)
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = feat.shape[0]
    losses = []
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    k = 0
    for ep in range(epochs):
        order = torch.randperm(n, generator=g, device="cuda")
        for i in range(steps_per_epoch):
            idx = order[i * batch:(i + 1) * batch]
            fb = feat[idx].contiguous()
            tb = target[idx].contiguous()
            # cosine decay of the learning rate
            lr_k = lr * 0.5 * (1.0 + np.cos(np.pi * k / total))
            want = log_every and (k % log_every == 0 or k == total - 1)
            l = tr.step(fb, tb, lr_k, want_loss=bool(want))
            if want:
                losses.append((k, l))
            k += 1
    return tr, losses


def save(path: str, w16: np.ndarray, b32: np.ndarray, **meta) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez_compressed(path, w16=w16, b32=b32, **{k: np.asarray(v) for k, v in meta.items()})


def load(path: str):
    d = np.load(path)
    return d["w16"], d["b32"]
