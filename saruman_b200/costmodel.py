"""Learned cost model of the autotuner.

A small tanh network predicts the banded kernel's log time per candidate
for a (read length, k, start-gap fraction, candidates) bin and a launch
shape.  It is trained on the GPU by the library's own kernels
(saru_mlp_loss_grad, saru_mlp_adam_step: forward, backward and Adam in
costmodel.cu) from autotuner measurements, and ranks the shapes of a new bin
so that the tuner times only the best few instead of the whole search space.
It changes only which launch shape runs, never which candidates are aligned
or their results.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np

N_FEATURES = 14
SWEEP = Path(__file__).resolve().parent / "tuning_sweep_b200.json"


def band_cells(m: int, k: int, so_frac: float) -> float:
    """Band cells per candidate: m(2k+1) without a start gap, m(4k+1) with."""
    return m * ((1.0 - so_frac) * (2 * k + 1) + so_frac * (4 * k + 1))


def features(m: int, k: int, so_frac: float, n: int, shape) -> np.ndarray:
    """The network's inputs for one bin and launch shape (all about 0..1)."""
    w, c, b = shape
    word64 = b == 64 or (b == 0 and k > 7)
    return np.array([
        math.log2(m) / 8.0, k / 16.0, so_frac, math.log2(max(n, 1)) / 21.0,
        float(w == 1), float(w == 2), float(w == 3), float(w in (0, 4)),
        float(c == 0), float(c == 2), float(c == 3),
        float(word64), math.log2(band_cells(m, k, so_frac)) / 16.0,
        math.log2(max(n, 1) / 32.0 / 148.0 + 1.0) / 10.0,  # tiles per SM
    ], np.float32)


def dataset(rows: list[dict]) -> tuple[np.ndarray, np.ndarray]:
    """Rows of a tuning sweep -> (features, log nanoseconds per candidate)."""
    X = np.stack([features(r["m"], r["k"], r["so_frac"], r["n"], tuple(r["shape"]))
                  for r in rows])
    y = np.array([math.log(r["ms"] * 1e6 / r["n"]) for r in rows], np.float32)
    return X, y


class CostModel:
    """The network's parameters on the device and its training loop."""

    def __init__(self, hidden=(32, 32), seed: int = 0, device: str = "cuda:0"):
        import torch
        import saruman_b200 as S
        self.S = S
        self.lib = S.load()
        self.device = device
        self.dims = (C.c_int32 * (len(hidden) + 2))(N_FEATURES, *hidden, 1)
        self.nl = len(hidden) + 1
        dims = list(self.dims)
        rng = np.random.default_rng(seed)
        parts = []
        for a, b in zip(dims[:-1], dims[1:]):  # Glorot-uniform weights, zero biases
            lim = math.sqrt(6.0 / (a + b))
            parts += [rng.uniform(-lim, lim, a * b), np.zeros(b)]
        p = np.concatenate(parts).astype(np.float32)
        assert p.size == self.lib.saru_mlp_param_count(self.dims, self.nl)
        self.params = torch.from_numpy(p).to(device)
        self.y_mean, self.y_std = 0.0, 1.0

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise self.S.SaruError(rc, self.S.last_error())

    def loss_grad(self, X: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
        """Loss and gradient of the raw network (no target scaling)."""
        import torch
        xs = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(self.device)
        ys = torch.from_numpy(np.ascontiguousarray(y, np.float32)).to(self.device)
        n = xs.shape[0]
        work = torch.empty(self.lib.saru_mlp_work_floats(self.dims, self.nl, n),
                           dtype=torch.float32, device=self.device)
        grad = torch.empty_like(self.params)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        self._check(self.lib.saru_mlp_loss_grad(self.dims, self.nl, self.params.data_ptr(),
                                                xs.data_ptr(), ys.data_ptr(), n,
                                                loss.data_ptr(), grad.data_ptr(),
                                                work.data_ptr(), None))
        torch.cuda.synchronize()
        return float(loss.item()), grad.cpu().numpy()

    def forward_raw(self, X: np.ndarray) -> np.ndarray:
        import torch
        xs = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(self.device)
        n = xs.shape[0]
        work = torch.empty(self.lib.saru_mlp_work_floats(self.dims, self.nl, n),
                           dtype=torch.float32, device=self.device)
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        self._check(self.lib.saru_mlp_forward(self.dims, self.nl, self.params.data_ptr(),
                                              xs.data_ptr(), n, out.data_ptr(), work.data_ptr(),
                                              None))
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def fit(self, X: np.ndarray, y: np.ndarray, steps: int = 3000, lr: float = 3e-3,
            lr_end: float = 3e-4) -> list[float]:
        """Full-batch Adam on the mean squared error of standardised targets,
        every step on the device; returns the loss every 100 steps."""
        import torch
        self.y_mean, self.y_std = float(np.mean(y)), float(np.std(y) + 1e-6)
        ys = torch.from_numpy(((y - self.y_mean) / self.y_std).astype(np.float32)).to(self.device)
        xs = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(self.device)
        n = xs.shape[0]
        work = torch.empty(self.lib.saru_mlp_work_floats(self.dims, self.nl, n),
                           dtype=torch.float32, device=self.device)
        grad = torch.empty_like(self.params)
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        count = self.params.numel()
        hist = []
        for step in range(1, steps + 1):
            a = lr * (lr_end / lr) ** ((step - 1) / max(steps - 1, 1))
            self._check(self.lib.saru_mlp_loss_grad(self.dims, self.nl, self.params.data_ptr(),
                                                    xs.data_ptr(), ys.data_ptr(), n,
                                                    loss.data_ptr(), grad.data_ptr(),
                                                    work.data_ptr(), None))
            self._check(self.lib.saru_mlp_adam_step(self.params.data_ptr(), grad.data_ptr(),
                                                    m.data_ptr(), v.data_ptr(), count, a, 0.9,
                                                    0.999, 1e-8, step, None))
            if step % 100 == 0 or step == 1:
                hist.append(float(loss.item()))
        return hist

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Predicted log nanoseconds per candidate."""
        return self.forward_raw(X) * self.y_std + self.y_mean

    def rank(self, m: int, k: int, so_frac: float, n: int, shapes) -> list:
        """Shapes from the predicted fastest to the slowest."""
        X = np.stack([features(m, k, so_frac, n, sh) for sh in shapes])
        order = np.argsort(self.predict(X), kind="stable")
        return [shapes[i] for i in order]


def trained_on_sweep(path: Path = SWEEP, steps: int = 3000, seed: int = 0) -> CostModel:
    """A model trained (on the GPU) on every row of a measured tuning sweep."""
    X, y = dataset(json.loads(Path(path).read_text())["rows"])
    net = CostModel(seed=seed)
    net.fit(X, y, steps=steps)
    return net
