"""Differentiable BD window: gradients of a smoothed pair-distance-histogram
loss of the final positions with respect to the pair-table values, the
bond-table values and the initial positions.

``Window`` drives the library's checkpointed forward window and its reverse
sweep (``mb2_window_forward`` / ``mb2_window_backward``) and the smoothed
histogram (``mb2_rdf_histogram`` / ``mb2_rdf_backward``); ``BDWindowLoss`` is
the ``torch.autograd.Function`` over them. Every kernel is the library's;
torch provides device memory and the autograd graph.

The loss is L = sum_b (g_b - g*_b)^2 with g_b = norm_b h_b, h_b the
Gaussian-smoothed count of non-excluded pairs at distance r_b (see
``include/marsb200.h``) and norm_b = V / (N (N - 1) / 2 * 4 pi r_b^2 dr).
The noise is fixed: Philox keyed on (seed, patch 0, absolute step), as in
every BD step of this library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .engine import Context, _p, _stream, setup_workload, step_params


@dataclass
class RdfSpec:
    bins: int = 100
    bin_width: float = 0.25
    r_max: float = 25.0
    sigma: float = 0.25

    def norm(self, n: int, volume: float) -> np.ndarray:
        r = (np.arange(self.bins) + 0.5) * self.bin_width
        return volume / (n * (n - 1) / 2.0 * 4.0 * math.pi * r * r * self.bin_width)


class Window:
    """A BD window of `steps` steps on a workload with bonds, angles and
    exclusions (``workloads.adjoint``), checkpointed every `checkpoint_every`."""

    def __init__(self, w, steps: int, checkpoint_every: int = 20, seed: int | None = None,
                 rdf: RdfSpec | None = None, device: str = "cuda:0"):
        self.w = w
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        self.rdf = rdf or RdfSpec()
        self.device = device
        self.ctx = Context(w.n, device=torch.device(device).index or 0)
        self.dev = setup_workload(self.ctx, w, device=device)
        if w.exclusions is not None and len(w.exclusions):
            off, nb = _exclusion_csr(w.exclusions, w.n)
            self.dev["excl_off"] = torch.from_numpy(off).to(device)
            self.dev["excl_nb"] = torch.from_numpy(nb).to(device)
            self.ctx.set_exclusions(self.dev["excl_off"], self.dev["excl_nb"], w.n)
        self.prm = step_params(w, seed=seed, bonds=self.dev.get("bonds"),
                               bond_idx=self.dev.get("bond_idx"), angles=self.dev.get("angles"),
                               angle_idx=self.dev.get("angle_idx"))
        self.prm.rebuild_period = max(self.prm.rebuild_period, 1)
        if self.prm.rebuild_period % self.every:
            self.prm.rebuild_period = self.every
        self.pair_sizes = [len(t.values) for t in w.pair_tables]
        self.bond_sizes = [len(t.values) for t in w.bond_tables]
        self.volume = float(np.prod(w.box_size))
        self.norm = torch.from_numpy(self.rdf.norm(w.n, self.volume)).to(device)

    # -- tables ----------------------------------------------------------------------
    def pair_values(self) -> torch.Tensor:
        return torch.from_numpy(np.concatenate([t.values for t in self.w.pair_tables])).to(
            self.device)

    def bond_values(self) -> torch.Tensor:
        return torch.from_numpy(np.concatenate([t.values for t in self.w.bond_tables])).to(
            self.device)

    def set_tables(self, pair_values: torch.Tensor, bond_values: torch.Tensor | None = None):
        pv = pair_values.detach().float().cpu().numpy()
        tabs, k = [], 0
        for t, size in zip(self.w.pair_tables, self.pair_sizes):
            tabs.append((pv[k:k + size], t.start, t.step_inv))
            k += size
        self.ctx.set_pair_tables(self.w.num_types, self.w.term_matrix, tabs)
        if bond_values is not None and self.bond_sizes:
            bv = bond_values.detach().float().cpu().numpy()
            tabs, k = [], 0
            for t, size in zip(self.w.bond_tables, self.bond_sizes):
                tabs.append((bv[k:k + size], t.start, t.step_inv))
                k += size
            self.ctx.set_bonded_tables(0, tabs)

    # -- passes ----------------------------------------------------------------------
    def forward(self, pos0: torch.Tensor, stream=None) -> torch.Tensor:
        """x_N of the window from x_0 (float32 [n, 4]); x_0 is not modified."""
        pos = pos0.detach().clone().contiguous()
        fe = torch.zeros_like(pos)
        self.ctx.check(self.ctx.lib.mb2_window_forward(
            self.ctx.h, _p(pos), _p(fe), _p(self.dev["type"]), self.w.n, 1, self.steps,
            self.every, C.byref(self.prm), _stream(stream)))
        return pos

    def checkpoints(self, stream=None) -> torch.Tensor:
        """Positions stored at the last forward window's checkpoints
        (ceil(steps / checkpoint_every) x n x 4, x_0 first)."""
        segs = (self.steps + self.every - 1) // self.every
        out = torch.empty((segs, self.w.n, 4), dtype=torch.float32, device=self.device)
        self.ctx.check(self.ctx.lib.mb2_window_checkpoints(
            self.ctx.h, _p(out), segs * self.w.n, _stream(stream)))
        return out

    def record_states(self, out: torch.Tensor | None):
        """Have each following backward write the states it differentiates
        (x_0 .. x_{steps-1}) into `out` (float32 [steps, n, 4] on the device),
        or stop with None."""
        if out is None:
            self.ctx.check(self.ctx.lib.mb2_window_record_states(self.ctx.h, None, 0))
            return
        if out.dtype != torch.float32 or tuple(out.shape) != (self.steps, self.w.n, 4):
            raise ValueError(f"record_states: float32 [{self.steps}, {self.w.n}, 4] expected")
        self._recorded = out
        self.ctx.check(self.ctx.lib.mb2_window_record_states(self.ctx.h, _p(out),
                                                             self.steps * self.w.n))

    def histogram(self, pos: torch.Tensor, stream=None) -> torch.Tensor:
        h = torch.zeros(self.rdf.bins, dtype=torch.float64, device=self.device)
        r = self.rdf
        self.ctx.check(self.ctx.lib.mb2_rdf_histogram(
            self.ctx.h, _p(pos), _p(self.dev["type"]), self.w.n, r.bins, r.bin_width, r.r_max,
            r.sigma, _p(h), _stream(stream)))
        return h

    def histogram_backward(self, pos: torch.Tensor, dldh: torch.Tensor, stream=None):
        g = torch.zeros_like(pos)
        r = self.rdf
        dl = dldh.to(torch.float64).contiguous()
        self.ctx.check(self.ctx.lib.mb2_rdf_backward(
            self.ctx.h, _p(pos), self.w.n, r.bins, r.bin_width, r.r_max, r.sigma, _p(dl), _p(g),
            _stream(stream)))
        return g

    def backward(self, grad_final: torch.Tensor, stream=None):
        """(dL/dx_0 [n, 4], dL/d pair values (float64), dL/d bond values (float64))."""
        g0 = torch.zeros_like(grad_final)
        gp = torch.zeros(sum(self.pair_sizes), dtype=torch.float64, device=self.device)
        gb = torch.zeros(max(sum(self.bond_sizes), 1), dtype=torch.float64, device=self.device)
        self.ctx.check(self.ctx.lib.mb2_window_backward(
            self.ctx.h, _p(grad_final.contiguous()), _p(g0), _p(gp), _p(gb), _stream(stream)))
        return g0, gp, gb[:sum(self.bond_sizes)]

    def loss_of(self, hist: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        return torch.sum((hist * self.norm - target) ** 2)

    def close(self):
        self.ctx.close()


class BDWindowLoss(torch.autograd.Function):
    """loss = sum_b (norm_b h_b(x_N) - target_b)^2, x_N the window's final
    positions; differentiable in the pair-table values, the bond-table values
    and the initial positions (float32 [n, 4]; the 4th column gets 0)."""

    @staticmethod
    def forward(ctx, pair_values, bond_values, pos0, window: Window, target):
        window.set_tables(pair_values, bond_values)
        pos_n = window.forward(pos0)
        hist = window.histogram(pos_n)
        ctx.window = window
        ctx.save_for_backward(pos_n, hist, target)
        return window.loss_of(hist, target)

    @staticmethod
    def backward(ctx, grad_loss):
        pos_n, hist, target = ctx.saved_tensors
        w = ctx.window
        dldh = grad_loss.to(torch.float64) * 2.0 * (hist * w.norm - target) * w.norm
        lam_n = w.histogram_backward(pos_n, dldh)
        g0, gp, gb = w.backward(lam_n)
        return gp.float(), gb.float(), g0, None, None


def _exclusion_csr(pairs: np.ndarray, n: int):
    """Symmetric CSR of excluded pairs (each stored under both endpoints)."""
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    a = np.concatenate([pairs[:, 0], pairs[:, 1]])
    b = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    off = np.zeros(n + 1, np.int32)
    np.add.at(off, a + 1, 1)
    return np.cumsum(off).astype(np.int32), b.astype(np.int32)
