"""Learned surrogate of the config-5 design problem: density -> spectrum.

A small convolutional encoder-decoder maps a 64 x 64 design density rho to
the complex transmission T(f) at 32 frequencies (wavelengths 1.4-1.7 um) of
the fixed 400 x 250 TE geometry (``workloads.config5_instance``). T is the
sum over the output line of the Ey DFT, divided by the same sum for the empty
design. The reference has no counterpart: it is the learned part of the
inverse-design stack, trained on spectra generated by the batched FDTD engine
(``batch.BatchTE``) and verified by its adjoint.

Network (NHWC, ``ARCH``; 1,750,562 parameters):
  encoder  conv3x3 1->32 (64x64), then stride-2 conv3x3 32->64 (32x32),
           64->128 (16x16), 128->256 (8x8), 256->128 (4x4), all ReLU;
  bottleneck  fully connected 2048 -> 512 (ReLU), read as 8 frequency
           positions x 64 channels;
  decoder  2x upsample, conv1x3 64->64 (ReLU) at 16 positions, 2x upsample,
           conv1x3 64->32 (ReLU) at 32 positions, conv1x1 32->2 = (Re T, Im T)
           per frequency.

BF16 weights and activations, FP32 accumulation, FP32 master weights and
Adam state. Every layer runs on the library's own kernels (the pfs_* entry
points of include/pfb200.h): im2col + tensor-core GEMM + bias/ReLU forward,
transposed GEMMs + col2im backward. PyTorch only holds the device buffers.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N


def _ceil32(n: int) -> int:
    return (n + 31) // 32 * 32


@dataclass
class Layer:
    kind: str             # "conv", "fc" or "up"
    cin: int = 0
    cout: int = 0
    kh: int = 1
    kw: int = 1
    stride: int = 1
    ph: int = 0
    pw: int = 0
    relu: bool = True
    # filled in by plan(): input / output spatial shape
    H: int = 0
    W: int = 0
    Ho: int = 0
    Wo: int = 0

    @property
    def K(self) -> int:
        return self.kh * self.kw * self.cin

    @property
    def Kp(self) -> int:
        return _ceil32(self.K)

    @property
    def coutp(self) -> int:  # output channels padded for the backward GEMMs
        return _ceil32(self.cout)


ARCH: List[Layer] = [
    Layer("conv", 1, 32, 3, 3, 1, 1, 1),
    Layer("conv", 32, 64, 3, 3, 2, 1, 1),
    Layer("conv", 64, 128, 3, 3, 2, 1, 1),
    Layer("conv", 128, 256, 3, 3, 2, 1, 1),
    Layer("conv", 256, 128, 3, 3, 2, 1, 1),
    Layer("fc", 2048, 512),
    Layer("up"),
    Layer("conv", 64, 64, 1, 3, 1, 0, 1),
    Layer("up"),
    Layer("conv", 64, 32, 1, 3, 1, 0, 1),
    Layer("conv", 32, 2, 1, 1, 1, 0, 0, relu=False),
]
N_FREQ = 32


def plan(arch: Sequence[Layer] = ARCH) -> List[Layer]:
    """Layer list with spatial shapes resolved from the 64 x 64 x 1 input."""
    out = []
    H, W, Cc = 64, 64, 1
    for L in arch:
        L = Layer(**L.__dict__)
        if L.kind == "conv":
            assert L.cin == Cc, (L, Cc)
            L.H, L.W = H, W
            L.Ho = (H + 2 * L.ph - L.kh) // L.stride + 1
            L.Wo = (W + 2 * L.pw - L.kw) // L.stride + 1
            H, W, Cc = L.Ho, L.Wo, L.cout
        elif L.kind == "fc":
            assert L.cin == H * W * Cc
            L.H, L.W, L.Ho, L.Wo = 1, 1, 1, 1
            H, W, Cc = 1, L.cout // 64, 64
        else:  # nearest 2x along the width (H = 1)
            assert H == 1
            L.H, L.W, L.Ho, L.Wo = H, W, H, 2 * W
            L.cin = L.cout = Cc
            W = 2 * W
        out.append(L)
    assert (H, W, Cc) == (1, N_FREQ, 2), (H, W, Cc)
    return out


def init_params(layers: Sequence[Layer], seed: int = 0) -> List[Tuple[np.ndarray, np.ndarray]]:
    """He-normal weights W[cout][K] (K order (ky, kx, c), matching im2col) and
    zero biases; the output layer starts small."""
    rng = np.random.default_rng(seed)
    params = []
    for L in layers:
        if L.kind == "up":
            params.append((None, None))
            continue
        std = math.sqrt(2.0 / L.K) if L.relu else 0.1 / math.sqrt(L.K)
        params.append((rng.standard_normal((L.cout, L.K)) * std, np.zeros(L.cout)))
    return params


def n_params(layers: Sequence[Layer]) -> int:
    return sum(L.cout * L.K + L.cout for L in layers if L.kind != "up")


class SurrogateNet:
    """The network on the GPU, for a fixed batch size (a multiple of 32).

    forward(x) takes a (B, 64, 64) BF16/FP32 torch tensor of inputs
    x = 2 rho - 1 and returns the (B, 32, 2) prediction; backward(dy) runs the
    reverse pass for an output gradient of that shape, filling the weight
    gradients and, with input_grad=True, returning dL/dx (B, 64, 64)."""

    def __init__(self, batch: int, params=None, seed: int = 0, device: str = "cuda",
                 t_mean=None, t_std=None):
        import torch
        if batch % 32:
            raise ValueError("batch must be a multiple of 32")
        self.torch = torch
        self.B = batch
        self.dev = device
        self.layers = plan()
        self.L = N.lib()
        # backward GEMMs read dY, the lowered input and W MN-major (no
        # transposed copies); PFB200_SURROGATE_TRANSPOSE=1 restores the copies
        self.mn_major = not os.environ.get("PFB200_SURROGATE_TRANSPOSE")
        # bias + activation in the forward GEMM's epilogue
        # (pfs_gemm_bf16_bias_act); PFB200_SURROGATE_UNFUSED=1 runs the
        # separate pass instead
        self.fused_epilogue = not os.environ.get("PFB200_SURROGATE_UNFUSED")
        if params is None:
            params = init_params(self.layers, seed)
        self._alloc(params)
        self.step_count = 0
        # the network predicts (T - t_mean) / t_std per (frequency, part)
        self.t_mean = np.zeros((N_FREQ, 2)) if t_mean is None else np.asarray(t_mean, np.float64)
        self.t_std = np.ones((N_FREQ, 2)) if t_std is None else np.asarray(t_std, np.float64)

    # ---- buffers ------------------------------------------------------- #
    def _alloc(self, params):
        t, B, dev = self.torch, self.B, self.dev
        f32, bf = t.float32, t.bfloat16
        self.w32, self.w16, self.b32, self.gw, self.gb = [], [], [], [], []
        self.m_w, self.v_w, self.m_b, self.v_b = [], [], [], []
        self.col, self.cpre, self.y32, self.y16 = [], [], [], []
        self.d16, self.dT, self.colT, self.wT, self.dcol, self.dx = [], [], [], [], [], []
        self.part = []
        for L, (Wn, bn) in zip(self.layers, params):
            if L.kind == "up":
                for lst in (self.w32, self.w16, self.b32, self.gw, self.gb, self.m_w, self.v_w,
                            self.m_b, self.v_b, self.col, self.cpre, self.d16, self.dT,
                            self.colT, self.wT, self.dcol, self.part):
                    lst.append(None)
                M = B * L.Ho * L.Wo
                self.y32.append(None)
                self.y16.append(t.zeros((M, L.cout), dtype=bf, device=dev))
                self.dx.append(t.zeros((B * L.H * L.W, L.cin), dtype=f32, device=dev))
                continue
            Kp, cp = L.Kp, L.coutp
            w = np.zeros((cp, Kp), np.float32)
            w[:L.cout, :L.K] = Wn
            b = np.zeros(cp, np.float32)
            b[:L.cout] = bn
            w32 = t.from_numpy(w).to(dev)
            self.w32.append(w32)
            self.w16.append(w32.to(bf))
            self.b32.append(t.from_numpy(b).to(dev))
            self.gw.append(t.zeros_like(w32))
            self.gb.append(t.zeros(cp, dtype=f32, device=dev))
            self.m_w.append(t.zeros_like(w32))
            self.v_w.append(t.zeros_like(w32))
            self.m_b.append(t.zeros(cp, dtype=f32, device=dev))
            self.v_b.append(t.zeros(cp, dtype=f32, device=dev))
            M = B * L.Ho * L.Wo
            self.col.append(t.zeros((M, Kp), dtype=bf, device=dev) if L.kind == "conv" else None)
            self.cpre.append(t.zeros((M, cp), dtype=f32, device=dev))
            self.y32.append(t.zeros((M, cp), dtype=f32, device=dev))
            self.y16.append(t.zeros((M, cp), dtype=bf, device=dev))
            self.d16.append(t.zeros((M, cp), dtype=bf, device=dev))
            # transposed copies only for the path that makes them
            tr = not self.mn_major
            self.dT.append(t.zeros((cp, M), dtype=bf, device=dev) if tr else None)
            self.colT.append(t.zeros((Kp, M), dtype=bf, device=dev) if tr else None)
            self.wT.append(t.zeros((Kp, cp), dtype=bf, device=dev) if tr else None)
            self.dcol.append(t.zeros((M, Kp), dtype=f32, device=dev))
            self.dx.append(t.zeros((B * L.H * L.W * L.cin,), dtype=f32, device=dev))
            rb = int(min(65535, max(1, M // 64)))
            self.part.append((t.zeros((rb, cp), dtype=f32, device=dev), rb))
        # split-K for the weight-gradient GEMMs (tiny output, K = all rows)
        self.splits = []
        wmax = 0
        for L in self.layers:
            if L.kind == "up":
                self.splits.append(1)
                continue
            M = B * L.Ho * L.Wo
            blocks = -(-L.coutp // 64) * -(-L.Kp // 64)
            sp = int(max(1, min(-(-296 // blocks), M // 512)))
            self.splits.append(sp)
            if sp > 1:
                wmax = max(wmax, sp * L.coutp * L.Kp)
        self.work = t.zeros(max(wmax, 1), dtype=f32, device=dev)
        self.x16 = t.zeros((B, 64, 64), dtype=bf, device=dev)
        self.gout = t.zeros((B * N_FREQ, 32), dtype=f32, device=dev)
        self.loss_parts = t.zeros(64, dtype=f32, device=dev)

    def _chk(self, rc):
        if rc != N.PF_OK:
            raise N.NativeError(rc, self.L.pfs_last_error().decode())

    @staticmethod
    def _p(x) -> int:
        return 0 if x is None else x.data_ptr()

    def _s(self) -> int:
        return self.torch.cuda.current_stream().cuda_stream

    # ---- forward ------------------------------------------------------- #
    def forward(self, x) -> "object":
        """x: (B, 64, 64) tensor (any float dtype) of 2 rho - 1."""
        L_, s = self.L, self._s()
        self.x16.copy_(x.reshape(self.B, 64, 64))
        inp = self.x16
        for li, L in enumerate(self.layers):
            if L.kind == "up":
                self._chk(L_.pfs_upsample2(self.B * L.H, L.W, L.cin, self._p(inp),
                                           self._p(self.y16[li]), s))
                inp = self.y16[li]
                continue
            M = self.B * L.Ho * L.Wo
            if L.kind == "conv":
                self._chk(L_.pfs_im2col(self.B, L.H, L.W, L.cin, L.kh, L.kw, L.stride, L.ph, L.pw,
                                        self._p(inp), self._p(self.col[li]), L.Kp, s))
                A = self.col[li]
            else:
                A = inp
            if self.fused_epilogue:
                self._chk(L_.pfs_gemm_bf16_bias_act(M, L.coutp, L.Kp, self._p(A), L.Kp,
                                                    self._p(self.w16[li]), L.Kp,
                                                    self._p(self.b32[li]), int(L.relu),
                                                    self._p(self.y32[li]), self._p(self.y16[li]),
                                                    L.coutp, s))
            else:
                self._chk(L_.pfs_gemm_bf16(M, L.coutp, L.Kp, self._p(A), L.Kp,
                                           self._p(self.w16[li]), L.Kp, self._p(self.cpre[li]),
                                           L.coutp, 1.0, 0.0, s))
                self._chk(L_.pfs_bias_act(M, L.coutp, self._p(self.cpre[li]),
                                          self._p(self.b32[li]), int(L.relu),
                                          self._p(self.y32[li]), self._p(self.y16[li]), s))
            inp = self.y16[li]
        self._last = li
        return self.y32[-1].view(self.B, N_FREQ, 32)[:, :, :2]

    # ---- backward ------------------------------------------------------ #
    def loss_grad(self, target) -> None:
        """MSE of the prediction against target (B, 32, 2) FP32; leaves the
        output gradient in place for backward(None)."""
        t32 = target.reshape(self.B * N_FREQ, 2).to(self.torch.float32).contiguous()
        self._target = t32
        self._chk(self.L.pfs_mse(self.B * N_FREQ, 2, 32, self._p(self.y32[-1]), self._p(t32),
                                 self._p(self.gout), self._p(self.loss_parts), 64, self._s()))

    def loss_value(self) -> float:
        return float(self.loss_parts.sum().item())

    def set_output_grad(self, dy) -> None:
        """Output gradient (B, 32, 2) FP32 for backward()."""
        self.gout.zero_()
        self.gout.view(self.B, N_FREQ, 32)[:, :, :2].copy_(dy)

    def backward(self, input_grad: bool = False):
        L_, s = self.L, self._s()
        dy = self.gout
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            first = li == 0
            if L.kind == "up":
                self._chk(L_.pfs_upsample2_bwd(self.B * L.H, L.W, L.cin, self._p(dy),
                                               self._p(self.dx[li]), s))
                dy = self.dx[li]
                continue
            M = self.B * L.Ho * L.Wo
            part, rb = self.part[li]
            self._chk(L_.pfs_act_bwd(M, L.coutp, self._p(dy), self._p(self.y32[li]), int(L.relu),
                                     0, self._p(self.d16[li]), self._p(self.gb[li]),
                                     self._p(part), rb, s))
            # weight gradient: dW = d^T col (K of the GEMM = M rows)
            A = self.col[li] if L.kind == "conv" else self.y16[li - 1]
            if self.mn_major:
                # the tensor cores read d and col as they lie (MN-major)
                self._chk(L_.pfs_gemm_bf16_ex(L.coutp, L.Kp, M, self._p(self.d16[li]), L.coutp,
                                              1, self._p(A), L.Kp, 1, self._p(self.gw[li]),
                                              L.Kp, 1.0, 0.0, self.splits[li],
                                              self._p(self.work), self.work.numel(), s))
                if first and not input_grad:
                    break
                # input gradient: dcol = d W, W read MN-major
                self._chk(L_.pfs_gemm_bf16_ex(M, L.Kp, L.coutp, self._p(self.d16[li]), L.coutp,
                                              0, self._p(self.w16[li]), L.Kp, 1,
                                              self._p(self.dcol[li]), L.Kp, 1.0, 0.0, 1, None,
                                              0, s))
            else:
                self._transposed_grads(li, L, M, A, s, not first or input_grad)
                if first and not input_grad:
                    break
            if L.kind == "conv":
                self._chk(L_.pfs_col2im(self.B, L.H, L.W, L.cin, L.kh, L.kw, L.stride, L.ph, L.pw,
                                        self._p(self.dcol[li]), L.Kp, self._p(self.dx[li]), s))
                dy = self.dx[li]
            else:
                dy = self.dcol[li]  # (B, 2048): the flattened NHWC input
        if input_grad:
            return self.dx[0].view(self.B, 64, 64)
        return None

    def _transposed_grads(self, li, L, M, A, s, need_dcol: bool) -> None:
        """dW (and dcol when need_dcol) through explicit BF16 transposes and
        K-major GEMMs: the form before MN-major operands, kept for comparison
        (PFB200_SURROGATE_TRANSPOSE=1)."""
        L_ = self.L
        self._chk(L_.pfs_transpose_bf16(M, L.coutp, self._p(self.d16[li]), L.coutp,
                                        self._p(self.dT[li]), M, s))
        self._chk(L_.pfs_transpose_bf16(M, L.Kp, self._p(A), L.Kp, self._p(self.colT[li]), M, s))
        self._chk(L_.pfs_gemm_bf16_splitk(L.coutp, L.Kp, M, self._p(self.dT[li]), M,
                                          self._p(self.colT[li]), M, self._p(self.gw[li]),
                                          L.Kp, 1.0, 0.0, self.splits[li],
                                          self._p(self.work), self.work.numel(), s))
        if not need_dcol:
            return
        self._chk(L_.pfs_transpose_bf16(L.coutp, L.Kp, self._p(self.w16[li]), L.Kp,
                                        self._p(self.wT[li]), L.coutp, s))
        self._chk(L_.pfs_gemm_bf16(M, L.Kp, L.coutp, self._p(self.d16[li]), L.coutp,
                                   self._p(self.wT[li]), L.coutp, self._p(self.dcol[li]),
                                   L.Kp, 1.0, 0.0, s))

    def adam_step(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8,
                  wd: float = 0.0) -> None:
        self.step_count += 1
        L_, s = self.L, self._s()
        for li, L in enumerate(self.layers):
            if L.kind == "up":
                continue
            self._chk(L_.pfs_adam(self.w32[li].numel(), self._p(self.w32[li]), self._p(self.gw[li]),
                                  self._p(self.m_w[li]), self._p(self.v_w[li]), lr, b1, b2, eps,
                                  self.step_count, wd, self._p(self.w16[li]), s))
            self._chk(L_.pfs_adam(self.b32[li].numel(), self._p(self.b32[li]), self._p(self.gb[li]),
                                  self._p(self.m_b[li]), self._p(self.v_b[li]), lr, b1, b2, eps,
                                  self.step_count, 0.0, 0, s))

    # ---- parameters ---------------------------------------------------- #
    def params(self) -> List[Tuple[np.ndarray, np.ndarray]]:
        out = []
        for li, L in enumerate(self.layers):
            if L.kind == "up":
                out.append((None, None))
                continue
            w = self.w32[li].cpu().numpy()[:L.cout, :L.K].astype(np.float64)
            b = self.b32[li].cpu().numpy()[:L.cout].astype(np.float64)
            out.append((w, b))
        return out

    def grads(self) -> List[Tuple[np.ndarray, np.ndarray]]:
        out = []
        for li, L in enumerate(self.layers):
            if L.kind == "up":
                out.append((None, None))
                continue
            out.append((self.gw[li].cpu().numpy()[:L.cout, :L.K].astype(np.float64),
                        self.gb[li].cpu().numpy()[:L.cout].astype(np.float64)))
        return out

    # ---- convenience --------------------------------------------------- #
    def predict(self, rho: np.ndarray) -> np.ndarray:
        """Complex T (n, 32) for densities rho (n, 64, 64), n padded up to
        whole batches internally."""
        t = self.torch
        rho = np.asarray(rho, np.float32).reshape(-1, 64, 64)
        out = np.empty((rho.shape[0], N_FREQ), np.complex128)
        for s0 in range(0, rho.shape[0], self.B):
            chunk = rho[s0:s0 + self.B]
            x = np.zeros((self.B, 64, 64), np.float32)
            x[:chunk.shape[0]] = 2.0 * chunk - 1.0
            y = self.forward(t.from_numpy(x).to(self.dev)).cpu().numpy().astype(np.float64)
            y = y * self.t_std + self.t_mean
            out[s0:s0 + chunk.shape[0]] = y[:chunk.shape[0], :, 0] + 1j * y[:chunk.shape[0], :, 1]
        return out

    def value_and_grad(self, rho: np.ndarray, objective: Callable) -> Tuple[np.ndarray, np.ndarray]:
        """Per-design objective(T) and its gradient with respect to rho, through
        the network (B designs at most). objective maps a torch complex (n, 32)
        tensor to (n,) values."""
        t = self.torch
        rho = np.asarray(rho, np.float32).reshape(-1, 64, 64)
        n = rho.shape[0]
        if n > self.B:
            raise ValueError("more designs than the batch size")
        x = np.zeros((self.B, 64, 64), np.float32)
        x[:n] = 2.0 * rho - 1.0
        y = self.forward(t.from_numpy(x).to(self.dev))[:n].detach().to(t.float64).cpu()
        yy = y.clone().requires_grad_(True)
        yd = yy * t.from_numpy(self.t_std) + t.from_numpy(self.t_mean)
        T = t.complex(yd[:, :, 0], yd[:, :, 1])
        v = objective(T)
        v.sum().backward()
        dy = t.zeros((self.B, N_FREQ, 2), dtype=t.float32)
        dy[:n] = yy.grad.to(t.float32)
        self.set_output_grad(dy.to(self.dev))
        dx = self.backward(input_grad=True)
        g = 2.0 * dx[:n].to(t.float64).cpu().numpy()  # x = 2 rho - 1
        return v.detach().numpy(), g

    def save(self, path: str) -> None:
        """The BF16 weights the kernels use (as uint16 bit patterns) and the
        FP32 biases, compressed."""
        arrs = {}
        for li, L in enumerate(self.layers):
            if L.kind == "up":
                continue
            w16 = self.w16[li][:L.cout, :L.K].contiguous().cpu()
            arrs[f"w{li}"] = w16.view(self.torch.int16).numpy().view(np.uint16)
            arrs[f"b{li}"] = self.b32[li][:L.cout].cpu().numpy()
        arrs["t_mean"] = self.t_mean
        arrs["t_std"] = self.t_std
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path: str, batch: int) -> "SurrogateNet":
        """A network with the weights and target normalisation saved by save()."""
        z = np.load(path)
        return cls(batch, params=cls.load_params(path), t_mean=z["t_mean"], t_std=z["t_std"])

    @staticmethod
    def load_params(path: str) -> List[Tuple[np.ndarray, np.ndarray]]:
        """Parameters saved by save(), as float64 arrays (BF16-exact weights)."""
        z = np.load(path)
        out = []
        for li, L in enumerate(plan()):
            if L.kind == "up":
                out.append((None, None))
                continue
            w = (z[f"w{li}"].astype(np.uint32) << 16).view(np.float32).astype(np.float64)
            out.append((w, z[f"b{li}"].astype(np.float64)))
        return out


# --------------------------------------------------------------------------- #
# Spectra from the FDTD engine
# --------------------------------------------------------------------------- #
def time_training_step(batch: int = 128, steps: int = 20, warmup: int = 3) -> float:
    """Milliseconds per training step (forward, loss, backward, AdamW) of the
    network on random inputs, by CUDA events after `warmup` steps."""
    import torch
    net = SurrogateNet(batch)
    x = torch.rand(batch, 64, 64, device="cuda") * 2 - 1
    t = torch.randn(batch, N_FREQ, 2, device="cuda")

    def step():
        net.forward(x)
        net.loss_grad(t)
        net.backward()
        net.adam_step(1e-3)
    for _ in range(warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def gemm_tflops(m: int, n: int, k: int, reps: int = 10, warmup: int = 3) -> float:
    """TFLOP/s (2mnk per call) of pfs_gemm_bf16 on random BF16 operands,
    C = A B^T with A m x k and B n x k, timed by CUDA events on the current
    stream after `warmup` calls."""
    import torch
    L = N.lib()
    st = torch.cuda.current_stream().cuda_stream
    A = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    B = torch.randn(n, k, device="cuda").to(torch.bfloat16)
    Cm = torch.empty(m, n, device="cuda")

    def run():
        rc = L.pfs_gemm_bf16(m, n, k, A.data_ptr(), k, B.data_ptr(), k, Cm.data_ptr(), n, 1.0,
                             0.0, st)
        if rc != N.PF_OK:
            raise N.NativeError(rc, L.pfs_last_error().decode())
    for _ in range(warmup):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    return 2.0 * m * n * k / (e0.elapsed_time(e1) / reps) / 1e9


class SpectrumGenerator:
    """Transmission spectra of the config-5 geometry for many designs, from
    one forward-only FDTD batch of `batch` copies of the geometry (designs
    are swapped in through the design-window coefficients).

    T(f) = sum_y F(f, y) / sum_y F_empty(f, y): the output-line Ey DFT
    summed over the line, divided by the empty design's (cladding only)."""

    def __init__(self, batch: int, precision: str = "float32", n_steps: int = 4000):
        import photonfdtd_b200 as pf
        from . import workloads as W
        from .batch import BatchTE
        self.W = W
        sim = W.config5_instance(pf, n_steps=n_steps, precision=precision)
        nx, ny = W.CONFIG5_SHAPE
        win = W.design_window_box(nx, ny, 64)
        self.batch = BatchTE([sim] * batch, [win] * batch, checkpoint_every=0)
        self.n = batch
        self.ny = ny
        empty = np.full(batch * 64 * 64, W.EPS_CLAD)
        self.batch.set_design_eps(empty)
        F = self.batch.forward()
        self.norm = F[:ny].sum(axis=0)  # instance 0, summed over the line
        self.cells = self.batch.ncell * self.batch.n_steps

    def eps_of(self, rho: np.ndarray) -> np.ndarray:
        W = self.W
        return W.EPS_CLAD + np.asarray(rho, np.float64) * (W.EPS_CORE - W.EPS_CLAD)

    def spectra(self, rho: np.ndarray) -> np.ndarray:
        """T (n, 32) complex for densities rho (n, 64, 64), n <= batch."""
        rho = np.asarray(rho, np.float64).reshape(-1, 64, 64)
        n = rho.shape[0]
        if n > self.n:
            raise ValueError("more designs than the batch holds")
        full = np.zeros((self.n, 64, 64))
        full[:n] = rho
        self.batch.set_design_eps(self.eps_of(full).ravel())
        F = self.batch.forward().reshape(self.n, self.ny, -1)
        return F[:n].sum(axis=1) / self.norm[None, :]

    def close(self):
        self.batch.close()


def densities(seeds: Sequence[int]) -> np.ndarray:
    """Config-4 densities (seeded Gaussian-filtered field through a sigmoid)."""
    from . import workloads as W
    return np.stack([W.config4_density(0, 64, seed_base=int(s)) for s in seeds])


# --------------------------------------------------------------------------- #
# Training and evaluation
# --------------------------------------------------------------------------- #
def train(net: SurrogateNet, x_all, t_all, epochs: int, lr: float = 2e-3, seed: int = 0,
          wd: float = 0.0, log: Optional[Callable[[str], None]] = None) -> List[float]:
    """Adam with a cosine learning-rate decay over `epochs` passes of the
    (x, target) pairs held on the GPU (x = 2 rho - 1, (n, 64, 64); target
    (n, 32, 2)). Returns the mean loss of every epoch."""
    import torch
    rng = np.random.default_rng(seed)
    n = int(x_all.shape[0])
    nb = n // net.B
    total = max(1, epochs * nb)
    hist = []
    k = 0
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(x_all.device)
        acc = torch.zeros((), dtype=torch.float32, device=x_all.device)
        for b in range(nb):
            idx = perm[b * net.B:(b + 1) * net.B]
            net.forward(x_all.index_select(0, idx))
            net.loss_grad(t_all.index_select(0, idx))
            acc += net.loss_parts.sum()
            net.backward()
            step_lr = 0.5 * lr * (1.0 + math.cos(math.pi * k / total))
            net.adam_step(step_lr, wd=wd)
            k += 1
        hist.append(float(acc.item()) / max(nb, 1))
        if log:
            log(f"epoch {ep + 1}/{epochs} loss {hist[-1]:.3e}")
    return hist


def spectrum_errors(pred: np.ndarray, true: np.ndarray) -> Dict[str, float]:
    """Relative L2 error per design, ||T_pred - T|| / ||T|| over the 32
    frequencies, summarised."""
    e = np.linalg.norm(pred - true, axis=1) / np.linalg.norm(true, axis=1)
    return {"mean": float(e.mean()), "median": float(np.median(e)),
            "p95": float(np.percentile(e, 95)), "max": float(e.max()),
            "frac_below_2pct": float(np.mean(e < 0.02)), "n": int(e.size)}


# --------------------------------------------------------------------------- #
# Inverse design: plain adjoint loop and surrogate-assisted loop
# --------------------------------------------------------------------------- #
def band_objective(T):
    """Two-band filter figure of merit per design, to maximise: mean |T|^2
    over the first 16 wavelengths (1.4-1.55 um) minus the mean over the last
    16 (1.55-1.7 um). Plain transmission is no target: the empty design has
    T = 1 by construction."""
    p = T.real ** 2 + T.imag ** 2
    return p[:, :16].mean(dim=1) - p[:, 16:].mean(dim=1)


class FDTDDesignProblem:
    """Exact objective and gradient of B config-5 designs by the batched FDTD
    engine and its adjoint (float32), plus forward-only verification."""

    def __init__(self, n_designs: int, objective: Callable = band_objective,
                 n_steps: int = 4000):
        import photonfdtd_b200 as pf
        from . import workloads as W
        from .batch import BatchTE
        self.W = W
        sim = W.config5_instance(pf, n_steps=n_steps)
        nx, ny = W.CONFIG5_SHAPE
        win = W.design_window_box(nx, ny, 64)
        self.n = n_designs
        self.ny = ny
        self.objective = objective
        self.batch = BatchTE([sim] * n_designs, [win] * n_designs)
        self.gen = SpectrumGenerator(n_designs, n_steps=n_steps)
        self.norm = self.gen.norm

    def _eps(self, rho):
        W = self.W
        return (W.EPS_CLAD + np.asarray(rho, np.float64) * (W.EPS_CORE - W.EPS_CLAD)).ravel()

    def value_grad_spectra(self, rho: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Objective, its gradient with respect to rho, and the spectra."""
        import torch
        from .batch import line_dft
        e = torch.tensor(self._eps(rho), requires_grad=True)
        F = line_dft(e, self.batch)
        norm = torch.from_numpy(self.norm)
        T = F.reshape(self.n, self.ny, -1).sum(dim=1) / norm
        v = self.objective(T)
        v.sum().backward()
        g = e.grad.numpy().reshape(self.n, 64, 64) * (self.W.EPS_CORE - self.W.EPS_CLAD)
        return v.detach().numpy(), g, T.detach().numpy()

    def value_and_grad(self, rho: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        v, g, _ = self.value_grad_spectra(rho)
        return v, g

    def spectra(self, rho: np.ndarray) -> np.ndarray:
        return self.gen.spectra(rho)

    def value(self, rho: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        import torch
        T = self.spectra(rho)
        return self.objective(torch.from_numpy(T)).numpy(), T

    def close(self):
        self.batch.close()
        self.gen.close()


class _Adam:
    """Adam ascent on a NumPy array (the design variables)."""

    def __init__(self, shape, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.m = np.zeros(shape)
        self.v = np.zeros(shape)
        self.t = 0
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    def ascend(self, x, g):
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return x + self.lr * mh / (np.sqrt(vh) + self.eps)


class SmoothDesign:
    """Design parameterisation on the manifold of the config-4 densities:
    rho = sigmoid(g / std(g)), g = F z F^T, with F the 64 x 64 matrix of the
    Gaussian filter (sigma = 3 cells, reflecting edges) and std taken per
    design. A unit-normal z reproduces config4_density exactly; every
    iterate keeps its smoothness and unit-spread statistics, the inputs the
    surrogate was trained on. grad_z is the exact chain rule (the filter
    transpose and the derivative of the normalisation)."""

    def __init__(self, sigma: float = 3.0, n: int = 64):
        from scipy.ndimage import gaussian_filter1d
        self.F = gaussian_filter1d(np.eye(n), sigma, axis=0, mode="reflect")

    def start(self, seeds: Sequence[int]) -> np.ndarray:
        return np.stack([np.random.default_rng(int(s)).standard_normal((64, 64)) for s in seeds])

    def _g(self, z):
        g = self.F @ z @ self.F.T
        return g, g.std(axis=(1, 2))[:, None, None]

    def rho(self, z: np.ndarray) -> np.ndarray:
        g, sd = self._g(z)
        return 1.0 / (1.0 + np.exp(-g / sd))

    def grad_z(self, z: np.ndarray, grad_rho: np.ndarray) -> np.ndarray:
        g, sd = self._g(z)
        r = 1.0 / (1.0 + np.exp(-g / sd))
        gh = grad_rho * r * (1.0 - r)                       # dJ/d(g / sd)
        gc = g - g.mean(axis=(1, 2), keepdims=True)
        n = g.shape[1] * g.shape[2]
        dg = gh / sd - gc * np.sum(gh * g, axis=(1, 2), keepdims=True) / (n * sd ** 3)
        return self.F.T @ dg @ self.F


def power_error(T_pred: np.ndarray, T_true: np.ndarray) -> np.ndarray:
    """Relative L2 error of the transmitted power |T|^2 over the frequencies,
    per design: the transmission the design objective is made of."""
    a, b = np.abs(T_pred) ** 2, np.abs(T_true) ** 2
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


class OnlineTuner:
    """Keeps the surrogate on the design trajectory: every FDTD spectrum the
    loop computes joins a buffer, and a few Adam steps train the network on
    batches mixing the newest buffer entries with replayed training pairs."""

    def __init__(self, net: SurrogateNet, replay_x=None, replay_t=None, lr: float = 5e-4,
                 steps: int = 20, seed: int = 0):
        self.net = net
        self.rx, self.rt = replay_x, replay_t
        self.lr, self.steps = lr, steps
        self.rng = np.random.default_rng(seed)
        self.bx: List[np.ndarray] = []
        self.bt: List[np.ndarray] = []

    def add(self, rho: np.ndarray, T: np.ndarray) -> None:
        tri = np.stack([T.real, T.imag], axis=-1)
        tn = (tri - self.net.t_mean) / self.net.t_std
        for r, t in zip(np.asarray(rho), tn):
            self.bx.append((2.0 * r - 1.0).astype(np.float32))
            self.bt.append(t.astype(np.float32))

    def tune(self) -> None:
        import torch
        net, B = self.net, self.net.B
        if not self.bx:
            return
        nb = len(self.bx)
        for _ in range(self.steps):
            k = min(nb, B // 2 if self.rx is not None else B)
            # newest half of the picks from the last 32 entries, the rest anywhere
            recent = self.rng.integers(max(0, nb - 32), nb, (k + 1) // 2)
            older = self.rng.integers(0, nb, k // 2)
            pick = np.concatenate([recent, older])
            x = torch.from_numpy(np.stack([self.bx[i] for i in pick])).to(net.dev)
            t = torch.from_numpy(np.stack([self.bt[i] for i in pick])).to(net.dev)
            if B - k > 0:
                if self.rx is not None:
                    idx = torch.from_numpy(self.rng.integers(0, self.rx.shape[0], B - k)).to(net.dev)
                    x = torch.cat([x, self.rx.index_select(0, idx).to(x.dtype)])
                    t = torch.cat([t, self.rt.index_select(0, idx).to(t.dtype)])
                else:
                    rep = torch.from_numpy(self.rng.integers(0, k, B - k)).to(net.dev)
                    x = torch.cat([x, x.index_select(0, rep)])
                    t = torch.cat([t, t.index_select(0, rep)])
            net.forward(x)
            net.loss_grad(t)
            net.backward()
            net.adam_step(self.lr)


def _sync():
    import torch
    torch.cuda.synchronize()


def trajectory_data(problem: FDTDDesignProblem, param: SmoothDesign, seeds: Sequence[int],
                    iters: int, lr: float = 0.05, every: int = 1,
                    log: Optional[Callable] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Training pairs from optimisation trajectories: the plain adjoint loop
    (plain_adjoint_loop's steps) run on problem.n designs at a time from the
    latent starts of `seeds`; every `every`-th iterate's density and its
    float32 FDTD spectrum (the forward pass of that iteration's gradient, so
    no extra FDTD run) are recorded. Returns (rho, T) stacked in the order
    [chunk of problem.n designs][recorded iteration][design]."""
    B = problem.n
    rhos, Ts = [], []
    for c0 in range(0, len(seeds) - B + 1, B):
        z = param.start(list(seeds[c0:c0 + B]))
        opt = _Adam(z.shape, lr)
        t0 = time.perf_counter()
        v = np.zeros(B)
        for it in range(iters):
            rho = param.rho(z)
            v, g, T = problem.value_grad_spectra(rho)
            if it % every == 0:
                rhos.append(rho.astype(np.float32))
                Ts.append(T)
            z = opt.ascend(z, param.grad_z(z, g))
        if log is not None:
            log(f"trajectories {c0}-{c0 + B - 1}: {iters} iterations in "
                f"{time.perf_counter() - t0:.1f} s, final objective {float(np.mean(v)):.4f}")
    return np.concatenate(rhos), np.concatenate(Ts)


def plain_adjoint_loop(problem: FDTDDesignProblem, param: SmoothDesign, z0: np.ndarray,
                       iters: int = 200, lr: float = 0.05) -> Dict:
    """Gradient ascent on the latent design z with the FDTD adjoint gradient
    every iteration (the plain method)."""
    z = np.array(z0, np.float64)
    opt = _Adam(z.shape, lr)
    hist = []
    _sync()
    t0 = time.perf_counter()
    for it in range(iters):
        v, g = problem.value_and_grad(param.rho(z))
        hist.append((time.perf_counter() - t0, it, float(np.mean(v))))
        z = opt.ascend(z, param.grad_z(z, g))
    v, _ = problem.value(param.rho(z))
    _sync()
    wall = time.perf_counter() - t0
    return {"z": z, "final": float(np.mean(v)), "final_each": v, "wall_s": wall,
            "history": hist, "fdtd_gradients": iters}


def surrogate_loop(problem: FDTDDesignProblem, net: SurrogateNet, param: SmoothDesign,
                   z0: np.ndarray, iters: int = 200, lr: float = 0.05,
                   verify_every: int = 10, max_error: float = 0.02,
                   tuner: Optional[OnlineTuner] = None, target: Optional[float] = None,
                   fallback_steps: int = 1, max_tries: int = 3, burst_lr: Optional[float] = None,
                   max_bursts: int = 1, grow: float = 1.0, max_burst_len: int = 80,
                   wall_budget: Optional[float] = None) -> Dict:
    """Surrogate-assisted gradient ascent on z with first-order model
    management (the additive-correction trust-region scheme of Alexandrov,
    Dennis, Lewis and Torczon, 1998). Each cycle:
      1. one plain step with the FDTD adjoint gradient g at the current
         design, whose forward pass also gives the verified objective there;
         the surrogate's gradient at the same design gives the correction
         d = g - g_sur, so the corrected model g_sur + d is exact to first
         order at that design;
      2. bursts of `verify_every` Adam steps on the corrected surrogate
         gradient (step size burst_lr, default lr), each verified by the FDTD
         forward run: a burst that raised the verified objective is kept and
         the next one follows (at most `max_bursts` kept per cycle); one that
         did not is rolled back (design and Adam state) and retried with half
         the step, at most `max_tries` rejections per cycle;
      3. fallback: the FDTD step of 1. also gives the true spectrum at its
         design, so the surrogate's power-transmission error there
         (power_error, mean over the designs) is known at the cost of one
         prediction; above `max_error` the cycle makes no burst and the next
         one takes `fallback_steps` plain FDTD steps, so while the network
         is off the loop is the plain adjoint loop.
    Every FDTD spectrum feeds `tuner` (online fine-tuning). Iterations are
    design updates: FDTD steps and kept surrogate steps count toward `iters`,
    rolled-back bursts do not. With `target`, records the wall-clock at which
    the best verified objective first reaches target - 1 % |target|.
    `grow` > 1 adapts the burst length: a kept burst multiplies it by grow
    (at most max_burst_len steps), a rejected one halves it (at least 2).
    `wall_budget` (seconds) ends the loop at the first cycle boundary past
    it, whatever `iters` says."""
    z = np.array(z0, np.float64)
    opt = _Adam(z.shape, lr)
    blr = lr if burst_lr is None else burst_lr
    best_z, best_v = z.copy(), -np.inf
    log = []
    n_fdtd_grad, n_verify, n_reject, n_kept = 0, 0, 0, 0
    reached = None
    n_plain = 1
    _sync()
    t0 = time.perf_counter()
    it = 0

    def note(v, zz):
        nonlocal best_v, best_z, reached
        if v > best_v:
            best_v, best_z = v, zz.copy()
        if target is not None and reached is None and best_v >= target - 0.01 * abs(target):
            reached = time.perf_counter() - t0

    burst_len = verify_every
    while it < iters:
        if wall_budget is not None and time.perf_counter() - t0 >= wall_budget:
            break
        # 1. plain FDTD steps; the last one's gradient corrects the surrogate
        for _ in range(min(n_plain, iters - it)):
            rho = param.rho(z)
            v, g, T = problem.value_grad_spectra(rho)
            n_fdtd_grad += 1
            cur_v = float(np.mean(v))
            note(cur_v, z)
            if tuner is not None:
                tuner.add(rho, T)
            _, g_sur = net.value_and_grad(rho, band_objective)
            delta = g - g_sur
            perr_fdtd = float(np.mean(power_error(net.predict(rho), T)))
            opt.lr = lr
            z = opt.ascend(z, param.grad_z(z, g))
            it += 1
        if it >= iters:
            break
        if perr_fdtd > max_error:  # 3. the surrogate sits this cycle out
            n_plain = fallback_steps
            log.append({"iter": it, "t": round(time.perf_counter() - t0, 3), "best": best_v,
                        "objective": cur_v, "bursts_kept": 0, "bursts_rejected": 0,
                        "power_error": perr_fdtd, "next_fdtd_steps": n_plain})
            if tuner is not None:
                tuner.tune()
            continue
        # 2. corrected surrogate bursts, each verified
        step, kept, rejected, perr, vt = blr, 0, 0, 0.0, cur_v
        while kept < max_bursts and rejected < max_tries and it < iters:
            saved = (z.copy(), opt.m.copy(), opt.v.copy(), opt.t)
            opt.lr = step
            n = min(burst_len, iters - it)
            for _ in range(n):
                _, gs = net.value_and_grad(param.rho(z), band_objective)
                z = opt.ascend(z, param.grad_z(z, gs + delta))
            rho = param.rho(z)
            v_true, T_true = problem.value(rho)
            n_verify += 1
            vt = float(np.mean(v_true))
            if tuner is not None:
                tuner.add(rho, T_true)
            perr = float(np.mean(power_error(net.predict(rho), T_true)))
            if vt > cur_v:
                cur_v = vt
                it += n
                n_kept += n
                kept += 1
                note(vt, z)
                if grow > 1.0:
                    burst_len = min(max_burst_len, int(round(burst_len * grow)))
            else:
                z, opt.m, opt.v, opt.t = saved
                step *= 0.5
                rejected += 1
                n_reject += 1
                if grow > 1.0:
                    burst_len = max(2, burst_len // 2)
        n_plain = fallback_steps if perr > max_error else 1
        log.append({"iter": it, "t": round(time.perf_counter() - t0, 3), "best": best_v,
                    "objective": cur_v, "bursts_kept": kept, "bursts_rejected": rejected,
                    "power_error": perr, "next_fdtd_steps": n_plain})
        if tuner is not None:
            tuner.tune()
    v_end, _ = problem.value(param.rho(z))
    n_verify += 1
    note(float(np.mean(v_end)), z)
    _sync()
    wall = time.perf_counter() - t0
    return {"z": best_z, "final": best_v, "wall_s": wall, "log": log,
            "fdtd_gradients": n_fdtd_grad, "fdtd_verifications": n_verify,
            "surrogate_steps_kept": n_kept, "surrogate_bursts_rejected": n_reject,
            "reached_target_s": reached}
