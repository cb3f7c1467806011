"""Learned cost model: a small MLP whose forward pass, backward pass, loss and Adam update run in
the engine's own CUDA kernels (csrc/mlp.cu, nnb_mlp_* in include/neonufft_gpu.h).

The network maps features of a (problem, configuration) pair to the logarithm of the measured
run time; neonufft_b200.tuner trains it on timings the engine generates and uses it to rank
configurations. No counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L
from .plan import check


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class MLP:
    """Fully connected network, tanh hidden layers, linear output, FP32 parameters on the GPU."""

    def __init__(self, widths: Sequence[int], seed: int = 0):
        import torch
        self.widths = [int(w) for w in widths]
        self.n_layers = len(self.widths) - 1
        self._cw = (C.c_int * len(self.widths))(*self.widths)
        n = C.c_int64(0)
        check(L.load().nnb_mlp_param_count(self.n_layers, self._cw, C.byref(n)))
        self.n_params = n.value
        rng = np.random.default_rng(seed)
        parts = []
        for l in range(1, len(self.widths)):
            n_in, n_out = self.widths[l - 1], self.widths[l]
            a = np.sqrt(6.0 / (n_in + n_out))
            parts.append(rng.uniform(-a, a, n_out * n_in))
            parts.append(np.zeros(n_out))
        self.params = torch.from_numpy(np.concatenate(parts).astype(np.float32)).cuda()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.step = 0

    def _acts(self, batch: int):
        import torch
        return torch.empty(sum(self.widths[1:]) * batch, dtype=torch.float32, device="cuda")

    def forward(self, x):
        """Returns (activation workspace, output view (batch x w_L))."""
        x = x.contiguous()
        batch = x.shape[0]
        acts = self._acts(batch)
        check(L.load().nnb_mlp_forward(self.n_layers, self._cw, self.params.data_ptr(),
                                       x.data_ptr(), batch, acts.data_ptr(), _stream()))
        out = acts[-batch * self.widths[-1]:].view(batch, self.widths[-1])
        return acts, out

    def backward(self, x, acts, dy) -> None:
        """Gradient of the parameters into self.grads for output gradient dy (batch x w_L)."""
        x = x.contiguous()
        batch = x.shape[0]
        dacts = acts.clone()
        dacts[-batch * self.widths[-1]:] = dy.reshape(-1)
        check(L.load().nnb_mlp_backward(self.n_layers, self._cw, self.params.data_ptr(),
                                        x.data_ptr(), acts.data_ptr(), dacts.data_ptr(), batch,
                                        self.grads.data_ptr(), _stream()))

    def mse(self, y, target):
        """(loss tensor of one float, dy) for the mean squared error of y against target."""
        import torch
        y = y.contiguous().reshape(-1)
        t = target.contiguous().reshape(-1).to(torch.float32)
        dy = torch.empty_like(y)
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        check(L.load().nnb_mlp_mse(y.data_ptr(), t.data_ptr(), y.numel(), dy.data_ptr(),
                                   loss.data_ptr(), _stream()))
        return loss, dy

    def adam(self, lr: float = 1e-2, beta1: float = 0.9, beta2: float = 0.999,
             eps: float = 1e-8) -> None:
        self.step += 1
        check(L.load().nnb_mlp_adam(self.n_params, self.params.data_ptr(), self.grads.data_ptr(),
                                    self.m.data_ptr(), self.v.data_ptr(), lr, beta1, beta2, eps,
                                    self.step, _stream()))

    def fit(self, x, y, epochs: int = 2000, lr: float = 1e-2) -> float:
        """Full-batch Adam on the mean squared error; returns the final loss."""
        loss = None
        for _ in range(epochs):
            acts, out = self.forward(x)
            loss, dy = self.mse(out, y)
            self.backward(x, acts, dy.view(out.shape))
            self.adam(lr)
        return float(loss.item()) if loss is not None else float("nan")

    def predict(self, x):
        return self.forward(x)[1].reshape(-1)


class CostModel:
    """Standardised features -> MLP -> log10 of the run time in milliseconds."""

    def __init__(self, n_features: int, hidden: Sequence[int] = (32, 32), seed: int = 0):
        self.net = MLP([n_features, *hidden, 1], seed=seed)
        self.mu = None
        self.sd = None

    def _norm(self, feats):
        import torch
        f = torch.as_tensor(np.asarray(feats, dtype=np.float32), device="cuda")
        return (f - self.mu) / self.sd

    def fit(self, feats, log_ms, epochs: int = 3000, lr: float = 5e-3) -> float:
        import torch
        f = torch.as_tensor(np.asarray(feats, dtype=np.float32), device="cuda")
        self.mu = f.mean(dim=0)
        self.sd = f.std(dim=0).clamp_min(1e-3)
        y = torch.as_tensor(np.asarray(log_ms, dtype=np.float32), device="cuda")
        return self.net.fit((f - self.mu) / self.sd, y.view(-1, 1), epochs=epochs, lr=lr)

    def predict(self, feats) -> np.ndarray:
        return self.net.predict(self._norm(feats)).cpu().numpy().astype(np.float64)

    def state(self) -> dict:
        """The trained model as plain lists (widths, parameters, feature standardisation)."""
        return {"widths": list(self.net.widths),
                "params": self.net.params.cpu().numpy().astype(np.float64).tolist(),
                "mu": self.mu.cpu().numpy().astype(np.float64).tolist(),
                "sd": self.sd.cpu().numpy().astype(np.float64).tolist()}

    @classmethod
    def from_state(cls, st: dict) -> "CostModel":
        """Rebuilds a trained model from state() (the network lives on the GPU)."""
        import torch
        widths = [int(w) for w in st["widths"]]
        m = cls(widths[0], hidden=widths[1:-1])
        params = np.asarray(st["params"], dtype=np.float32)
        if params.size != m.net.n_params:
            raise ValueError("parameter count does not match the widths")
        m.net.params.copy_(torch.from_numpy(params))
        m.mu = torch.as_tensor(np.asarray(st["mu"], dtype=np.float32), device="cuda")
        m.sd = torch.as_tensor(np.asarray(st["sd"], dtype=np.float32), device="cuda")
        return m
