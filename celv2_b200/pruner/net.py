"""The pruner network's parameters and its training loop on the GPU.

Every computation runs in the library's kernels (celv2_pruner_forward / _backward / _bce / _adam,
csrc/pruner.cu); torch tensors only provide the device memory and the stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import engine as E

# (name, shape) in parameter order, as include/celv2_pruner.h lays them out
SHAPES = [("W1", (16, 9)), ("b1", (16,)), ("W2", (32, 144)), ("b2", (32,)), ("W3", (32, 288)), ("b3", (32,)),
          ("W4", (64, 632)), ("b4", (64,)), ("W5", (E.PRUNER_OUTPUTS, 64)), ("b5", (E.PRUNER_OUTPUTS,))]
assert sum(int(np.prod(s)) for _, s in SHAPES) == E.PRUNER_PARAMS


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (fan-in = the row length), zero biases; the output layer scaled down."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name[0] == "W":
            w = rng.normal(0.0, np.sqrt(2.0 / shape[1]), shape)
            if name == "W5":
                w *= 0.1
            parts.append(w.reshape(-1))
        else:
            parts.append(np.zeros(shape).reshape(-1))
    return np.concatenate(parts).astype(np.float32)


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


class Trainer:
    """Adam on the weighted binary cross-entropy, minibatches of `batch` samples on one GPU."""

    def __init__(self, batch: int, device: int = 0, lr: float = 2e-3, weight_decay: float = 1e-4,
                 params: np.ndarray | None = None, seed: int = 0):
        import torch

        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        self.batch = batch
        self.lr, self.wd = lr, weight_decay
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        z = lambda n: torch.zeros(n, dtype=torch.float32, device=self.dev)  # noqa: E731
        self.g, self.m, self.v = z(E.PRUNER_PARAMS), z(E.PRUNER_PARAMS), z(E.PRUNER_PARAMS)
        self.acts = z(batch * E.PRUNER_ACTS)
        self.work = z(batch * E.PRUNER_WORK)
        self.dlogits = z(batch * E.PRUNER_OUTPUTS)
        self.loss = z(1)
        self.steps = 0

    def _stream(self) -> C.c_void_p:
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def logits(self, x) -> "torch.Tensor":
        """Forward pass of x (n <= batch samples, a float32 device tensor n x FEATURES)."""
        n = x.shape[0]
        E._check(E.library().celv2_pruner_forward(_ptr(self.p), _ptr(x), n, _ptr(self.acts), self._stream()))
        off = n * (E.PRUNER_ACTS - E.PRUNER_OUTPUTS)
        return self.acts[off:off + n * E.PRUNER_OUTPUTS].view(n, E.PRUNER_OUTPUTS)

    def step(self, x, y, w) -> None:
        """One Adam step on the minibatch (device tensors n x FEATURES, n x OUTPUTS, n x OUTPUTS)."""
        lib = E.library()
        n = x.shape[0]
        st = self._stream()
        z = self.logits(x)
        E._check(lib.celv2_pruner_bce(_ptr(z), _ptr(y), _ptr(w), n, _ptr(self.dlogits), _ptr(self.loss), st))
        E._check(lib.celv2_pruner_backward(_ptr(self.p), n, _ptr(self.acts), _ptr(self.dlogits), _ptr(self.work),
                                           _ptr(self.g), st))
        self.steps += 1
        E._check(lib.celv2_pruner_adam(_ptr(self.p), _ptr(self.g), _ptr(self.m), _ptr(self.v), E.PRUNER_PARAMS,
                                       self.lr, 0.9, 0.999, 1e-8, self.wd, self.steps, st))

    def take_loss(self) -> float:
        """The summed loss since the last call (synchronises)."""
        v = float(self.loss.item())
        self.loss.zero_()
        return v

    def params(self) -> np.ndarray:
        return self.p.detach().cpu().numpy().copy()

    def predict(self, x, chunk: int | None = None):
        """Sigmoid outputs for all of x (a device tensor), in chunks of the batch size (host array)."""
        out = []
        chunk = chunk or self.batch
        for i in range(0, x.shape[0], chunk):
            out.append(self.torch.sigmoid(self.logits(x[i:i + chunk])).cpu().numpy())
        return np.concatenate(out)
