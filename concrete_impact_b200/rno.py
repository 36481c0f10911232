"""Recurrent neural operator (RNO) material surrogate on the tensor-core kernels.

A recurrent MLP maps, per macro material point and time step, the macro strain, its rate
and a 6-component latent state to the homogenised stress and the latent rate; the latent
state advances with forward Euler, z' = z + (dt / tau_ref) zdot, as the reference's RVE-RNO
does (src/concrete_impact/nn/models/rve_rno.py:383-387).  The network is
18 -> 128 -> 128 -> 128 (GELU) -> 12 with bf16 weights and activations and fp32
accumulation; every matrix product runs in the tcgen05 GEMM of ``csrc/mlp.cu``
(``cib_mlp_gemm``) and every other step in the kernels of ``csrc/rno.cu``.

Training follows the reference's batched path rollout (all paths of a batch advance per
time index, src/concrete_impact/nn/training/rve_rno.py:113-197) with a normalised stress
MSE, Adam, and truncated backpropagation through time over windows of ``tbptt_steps``
(the latent state is carried across windows without gradient).  One window's forward,
backward, weight gradients and Adam update are captured once in a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .mlp import EPI_BIAS_F32, EPI_BIAS_GELU, EPI_F32, EPI_GELU_BWD, EPI_PARTIAL, gemm, splitk_reduce

IN_REAL, IN_PAD, OUT_REAL, OUT_PAD = 18, 32, 12, 16


@dataclass(frozen=True)
class RNOConfig:
    """Surrogate and training settings."""

    hidden: int = 128
    tau_ref: float = 1.0e-3
    learning_rate: float = 1.0e-3
    batch_paths: int = 512
    tbptt_steps: int = 50
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1.0e-8
    seed: int = 0


@dataclass(frozen=True)
class RNOScales:
    """Normalisation: strain, strain rate and stress are divided by these scales."""

    strain: float
    rate: float
    stress: float

    @staticmethod
    def from_data(strain: torch.Tensor, rate: torch.Tensor, stress: torch.Tensor) -> RNOScales:
        def s(x: torch.Tensor) -> float:
            v = float(x.double().pow(2).mean().sqrt().item())
            return v if v > 0 else 1.0

        return RNOScales(s(strain), s(rate), s(stress))


@dataclass
class RNODataset:
    """Macro paths on the device: strain and stress at steps 0..T (step 0 at rest) and the
    time steps dt (P, T)."""

    strain: torch.Tensor  # (P, T + 1, 6)
    stress: torch.Tensor  # (P, T + 1, 6)
    dt: torch.Tensor  # (P, T)

    @property
    def paths(self) -> int:
        return int(self.strain.shape[0])

    @property
    def steps(self) -> int:
        return int(self.dt.shape[1])

    def rates(self) -> torch.Tensor:
        return (self.strain[:, 1:] - self.strain[:, :-1]) / self.dt[..., None]


@dataclass
class _Layer:
    w: torch.Tensor  # fp32 master (out, in_pad)
    b: torch.Tensor  # fp32 (out,)
    wb: torch.Tensor  # bf16 (out, in_pad)
    wt: torch.Tensor  # bf16 (in_pad, out)
    mw: torch.Tensor
    vw: torch.Tensor
    mb: torch.Tensor
    vb: torch.Tensor
    gw: torch.Tensor
    gb: torch.Tensor


def _check(code: int, what: str) -> None:
    _native.check(code, what)


class RNOSurrogate:
    """The surrogate's parameters, optimiser state and device work buffers."""

    def __init__(self, config: RNOConfig = RNOConfig(), scales: RNOScales | None = None) -> None:
        self.device = _native.require_cuda()
        self.lib = _native.load_library()
        self.config = config
        self.scales = scales or RNOScales(1.0, 1.0, 1.0)
        h = config.hidden
        if h % 16 != 0 or h > 128:
            raise ValueError("hidden width must be a multiple of 16 and at most 128")
        g = torch.Generator().manual_seed(config.seed)
        dims = [(h, IN_PAD, IN_REAL), (h, h, h), (h, h, h), (OUT_PAD, h, h)]
        self.layers: list[_Layer] = []
        for out, inp, fan_in in dims:
            bound = 1.0 / math.sqrt(fan_in)
            w = (torch.rand((out, inp), generator=g) * 2 - 1) * bound
            b = (torch.rand((out,), generator=g) * 2 - 1) * bound
            if inp == IN_PAD:
                w[:, IN_REAL:] = 0.0
            if out == OUT_PAD:
                w[OUT_REAL:] = 0.0
                b[OUT_REAL:] = 0.0
            self.layers.append(self._make_layer(w, b))
        self.step = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.learning_rate = float(config.learning_rate)
        self.divergences = 0  # epochs rolled back by the training divergence guard
        # fused window kernels (one CTA per 128 paths for the whole window) for width 128
        self.fused = h == 128
        self.skip: torch.Tensor | None = None  # 6x6 normalised elastic skip, fused path only
        self._structs: dict = {}
        self._window: dict | None = None
        self._graph: torch.cuda.CUDAGraph | None = None

    def _make_layer(self, w: torch.Tensor, b: torch.Tensor) -> _Layer:
        dev = self.device
        w = w.to(dev).contiguous()
        b = b.to(dev).contiguous()
        z = torch.zeros_like
        return _Layer(w, b, w.to(torch.bfloat16).contiguous(), w.T.contiguous().to(torch.bfloat16), z(w), z(w), z(b), z(b),
                      z(w), z(b))  # fmt: skip

    # -- parameters ---------------------------------------------------------------------
    def state_dict(self) -> dict[str, torch.Tensor]:
        out: dict[str, torch.Tensor] = {}
        for i, L in enumerate(self.layers):
            out[f"layers.{i}.weight"] = L.w.detach().cpu().clone()
            out[f"layers.{i}.bias"] = L.b.detach().cpu().clone()
        out["scales"] = torch.tensor([self.scales.strain, self.scales.rate, self.scales.stress], dtype=torch.float64)
        if self.skip is not None:
            out["skip"] = self.skip.detach().cpu().clone()
        return out

    def load_state_dict(self, state: dict[str, torch.Tensor]) -> None:
        for i, L in enumerate(self.layers):
            L.w.copy_(state[f"layers.{i}.weight"].to(self.device))
            L.b.copy_(state[f"layers.{i}.bias"].to(self.device))
            L.wb.copy_(L.w.to(torch.bfloat16))
            L.wt.copy_(L.w.T.to(torch.bfloat16))
        s = state["scales"].tolist()
        self.scales = RNOScales(*s)
        self.skip = state["skip"].to(self.device).contiguous() if "skip" in state else None
        self._structs = {}
        self._graph = None

    def checkpoint(self) -> dict[str, torch.Tensor]:
        """Weights, scales, skip term, Adam moments, step counter and step size (host
        tensors): everything training needs to resume, as the reference's training loop
        checkpoints model and optimizer together (src/concrete_impact/nn/training/rve_rno.py:997-1012)."""
        out = self.state_dict()
        out["tau_ref"] = torch.tensor(self.config.tau_ref, dtype=torch.float64)
        out["learning_rate"] = torch.tensor(self.learning_rate, dtype=torch.float64)
        out["adam.step"] = self.step.detach().cpu().clone()
        for i, L in enumerate(self.layers):
            for name in ("mw", "vw", "mb", "vb"):
                out[f"adam.{i}.{name}"] = getattr(L, name).detach().cpu().clone()
        return out

    def load_checkpoint(self, state: dict[str, torch.Tensor]) -> None:
        """Restore a ``checkpoint``; training continues where it stopped."""
        self.load_state_dict(state)
        self.step.copy_(state["adam.step"].to(self.device))
        for i, L in enumerate(self.layers):
            for name in ("mw", "vw", "mb", "vb"):
                getattr(L, name).copy_(state[f"adam.{i}.{name}"].to(self.device))
        self.set_learning_rate(float(state["learning_rate"]))

    # -- window buffers ---------------------------------------------------------------
    def _buffers(self, T: int, B: int) -> dict:
        if self._window is not None and self._window["T"] == T and self._window["B"] == B:
            return self._window
        dev, h = self.device, self.config.hidden
        R = T * B
        Rp = ((R + 63) // 64) * 64  # transposed buffers: K of the weight-gradient GEMMs, zero-padded
        f32, bf = torch.float32, torch.bfloat16

        def e(*shape, dtype=f32):
            return torch.zeros(shape, dtype=dtype, device=dev)

        splits = max(1, min(64, Rp // 512))
        self._window = {
            "T": T, "B": B, "R": R, "Rp": Rp, "splits": splits,
            "strain": e(T, B, 6), "rate": e(T, B, 6), "target": e(T, B, 6), "coef": e(T, B), "z": e(T + 1, B, 6),
            "X": e(T, B, IN_PAD, dtype=bf), "Xt": e(IN_PAD, Rp, dtype=bf),
            "Z": [e(T, B, h) for _ in range(3)], "H": [e(T, B, h, dtype=bf) for _ in range(3)],
            "Ht": [e(h, Rp, dtype=bf) for _ in range(3)],
            "Y": e(T, B, OUT_PAD), "gY": e(T, B, 6),
            "loss_part": torch.zeros((T, (B + 127) // 128), dtype=torch.float64, device=dev),
            "dY": e(B, OUT_PAD, dtype=bf), "dYt": e(OUT_PAD, Rp, dtype=bf),
            "dZ": [e(B, h, dtype=bf) for _ in range(3)], "dZt": [e(h, Rp, dtype=bf) for _ in range(3)],
            "dX": e(B, IN_PAD), "dz": [e(B, 6), e(B, 6)],
            "partial": e(splits * h, h),
        }  # fmt: skip
        self._graph = None
        return self._window

    # -- one window ---------------------------------------------------------------------
    def _window_struct(self, w: dict, with_loss: bool) -> _native.RNOWindowC:
        """C descriptor of a window's buffers (kept alive with the window)."""
        key = (id(w), with_loss)
        if key in self._structs:
            return self._structs[key]
        c = _native.RNOWindowC()
        c.B, c.T, c.hidden = w["B"], w["T"], self.config.hidden
        c.ldt = w["Rp"]
        c.loss_scale = 1.0 / float(w["B"] * w["T"] * 6)
        c.strain, c.rate, c.coef = w["strain"].data_ptr(), w["rate"].data_ptr(), w["coef"].data_ptr()
        c.target = w["target"].data_ptr() if with_loss else None
        c.z = w["z"].data_ptr()
        for i, L in enumerate(self.layers):
            c.W[i], c.Wt[i], c.bias[i] = L.wb.data_ptr(), L.wt.data_ptr(), L.b.data_ptr()
        c.skip = None if self.skip is None else self.skip.data_ptr()
        for i in range(3):
            c.Z[i], c.Ht[i], c.dZt[i] = w["Z"][i].data_ptr(), w["Ht"][i].data_ptr(), w["dZt"][i].data_ptr()
        c.Xt = w["Xt"].data_ptr()
        c.stress = None
        c.gS = w["gY"].data_ptr() if with_loss else None
        c.loss_part = w["loss_part"].data_ptr() if with_loss else None
        c.dYt = w["dYt"].data_ptr()
        c.err = self.err.data_ptr()
        self._structs = {k: v for k, v in self._structs.items() if k[0] == id(w)}
        self._structs[key] = c
        return c

    def _forward(self, w: dict, with_loss: bool) -> None:
        if self.fused:
            c = self._window_struct(w, with_loss)
            _check(self.lib.cib_rno_window_forward(ctypes.byref(c), _native.stream_ptr()), "cib_rno_window_forward")
            return
        if self.skip is not None:
            raise ValueError("the elastic skip term needs the fused kernels (hidden width 128)")
        T, B, R = w["T"], w["B"], w["R"]
        L = self.layers
        lib = self.lib
        sp = _native.stream_ptr()
        scale = 1.0 / float(B * T * 6)
        for t in range(T):
            _check(lib.cib_rno_input(B, w["strain"][t].data_ptr(), w["rate"][t].data_ptr(), w["z"][t].data_ptr(),
                                     w["X"][t].data_ptr(), w["Xt"].data_ptr(), w["Rp"], t * B, sp), "cib_rno_input")  # fmt: skip
            a = w["X"][t]
            for i in range(3):
                gemm(EPI_BIAS_GELU, a, L[i].wb, bias=L[i].b, z=w["Z"][i][t], h=w["H"][i][t], ht=w["Ht"][i],
                     row_offset=t * B, err=self.err)  # fmt: skip
                a = w["H"][i][t]
            gemm(EPI_BIAS_F32, a, L[3].wb, bias=L[3].b, c=w["Y"][t], err=self.err)
            _check(lib.cib_rno_forward_tail(
                B, w["Y"][t].data_ptr(), w["target"][t].data_ptr() if with_loss else None, w["coef"][t].data_ptr(),
                w["z"][t].data_ptr(), w["z"][t + 1].data_ptr(), w["gY"][t].data_ptr() if with_loss else None,
                scale, w["loss_part"][t].data_ptr() if with_loss else None, sp), "cib_rno_forward_tail")  # fmt: skip

    def _backward(self, w: dict) -> None:
        T, B, R = w["T"], w["B"], w["R"]
        L = self.layers
        lib = self.lib
        sp = _native.stream_ptr()
        if self.fused:
            c = self._window_struct(w, True)
            _check(lib.cib_rno_window_backward(ctypes.byref(c), sp), "cib_rno_window_backward")
        else:
            self._backward_steps(w)
        self._weight_gradients(w)

    def _backward_steps(self, w: dict) -> None:
        T, B, R = w["T"], w["B"], w["R"]
        L = self.layers
        lib = self.lib
        sp = _native.stream_ptr()
        dz_next, dz = w["dz"]
        dz_next.zero_()
        for t in range(T - 1, -1, -1):
            _check(lib.cib_rno_backward_head(B, w["gY"][t].data_ptr(), w["coef"][t].data_ptr(), dz_next.data_ptr(),
                                             w["dY"].data_ptr(), w["dYt"].data_ptr(), w["Rp"], t * B, sp),
                   "cib_rno_backward_head")  # fmt: skip
            grad = w["dY"]
            for i in (2, 1, 0):
                gemm(EPI_GELU_BWD, grad, L[i + 1].wt, n=self.config.hidden, z=w["Z"][i][t], h=w["dZ"][i],
                     ht=w["dZt"][i], row_offset=t * B, err=self.err)  # fmt: skip
                grad = w["dZ"][i]
            gemm(EPI_F32, grad, L[0].wt, c=w["dX"], err=self.err)
            _check(lib.cib_rno_backward_tail(B, dz_next.data_ptr(), w["dX"].data_ptr(), dz.data_ptr(), sp),
                   "cib_rno_backward_tail")  # fmt: skip
            dz_next, dz = dz, dz_next

    def _weight_gradients(self, w: dict) -> None:
        """Weight and bias gradients over all rows of the window (split-K GEMMs)."""
        R = w["R"]
        L = self.layers
        lib = self.lib
        sp = _native.stream_ptr()
        h = self.config.hidden
        ins = [w["Xt"], w["Ht"][0], w["Ht"][1], w["Ht"][2]]
        outs = [w["dZt"][0], w["dZt"][1], w["dZt"][2], w["dYt"]]
        for i in range(4):
            m = L[i].w.shape[0]
            n = L[i].w.shape[1]
            part = w["partial"][: w["splits"] * m]
            gemm(EPI_PARTIAL, outs[i], ins[i], c=part, splits=w["splits"], err=self.err, rows=m)
            splitk_reduce(part.view(w["splits"], m, n) if n == h else part, w["splits"], m, n, L[i].gw)
            _check(lib.cib_row_sum_bf16(m, R, outs[i].data_ptr(), w["Rp"], L[i].gb.data_ptr(), sp), "cib_row_sum_bf16")

    def _adam(self) -> None:
        lib, sp, c = self.lib, _native.stream_ptr(), self.config
        _check(lib.cib_counter_increment(self.step.data_ptr(), sp), "cib_counter_increment")
        for L in self.layers:
            out, inp = L.w.shape
            _check(lib.cib_adam_step(out, inp, L.w.data_ptr(), L.gw.data_ptr(), L.mw.data_ptr(), L.vw.data_ptr(),
                                     self.learning_rate, c.beta1, c.beta2, c.eps, self.step.data_ptr(), L.wb.data_ptr(),
                                     inp, L.wt.data_ptr(), out, sp), "cib_adam_step")  # fmt: skip
            _check(lib.cib_adam_step(1, out, L.b.data_ptr(), L.gb.data_ptr(), L.mb.data_ptr(), L.vb.data_ptr(),
                                     self.learning_rate, c.beta1, c.beta2, c.eps, self.step.data_ptr(), None, 0, None, 0,
                                     sp), "cib_adam_step")  # fmt: skip
        # padded rows/columns stay zero: their gradients are identically zero

    def set_learning_rate(self, lr: float) -> None:
        """Change Adam's step size; the captured training graph holds it as a launch
        argument, so it is captured again at the next replay."""
        if float(lr) != self.learning_rate:
            self.learning_rate = float(lr)
            self._graph = None

    def window_step(self, T: int, B: int, train: bool = True) -> None:
        """Forward (+ backward, gradients and Adam when ``train``) on the loaded window."""
        w = self._buffers(T, B)
        self._forward(w, True)
        if train:
            self._backward(w)
            self._adam()

    def window_gradients(self, T: int, B: int) -> None:
        """Forward and backward on the loaded window without the optimiser step."""
        w = self._buffers(T, B)
        self._forward(w, True)
        self._backward(w)

    def gradients(self) -> list[tuple[torch.Tensor, torch.Tensor]]:
        """(weight, bias) gradients of the last backward pass, fp32, padded shapes."""
        return [(L.gw, L.gb) for L in self.layers]

    def load_window(self, strain, rate, target, coef, z0) -> None:
        """Copy a window (time-major (T, B, 6) normalised inputs, (T, B) coefficients,
        (B, 6) initial latent) into the static buffers."""
        T, B = int(strain.shape[0]), int(strain.shape[1])
        w = self._buffers(T, B)
        w["strain"].copy_(strain)
        w["rate"].copy_(rate)
        w["target"].copy_(target)
        w["coef"].copy_(coef)
        w["z"][0].copy_(z0)

    def window_loss(self) -> float:
        """Mean squared normalised stress error of the last forward window."""
        w = self._window
        return float(w["loss_part"].sum().item()) / float(w["B"] * w["T"] * 6)

    # -- training -----------------------------------------------------------------------
    def _snapshot(self) -> list[torch.Tensor]:
        """Device copies of the weights, Adam moments and step counter."""
        out = [self.step.clone()]
        for L in self.layers:
            out += [L.w.clone(), L.b.clone(), L.mw.clone(), L.vw.clone(), L.mb.clone(), L.vb.clone()]
        return out

    def _restore(self, snap: list[torch.Tensor]) -> None:
        """Copy a snapshot back in place (the captured training graph keeps its buffers)."""
        self.step.copy_(snap[0])
        for i, L in enumerate(self.layers):
            w, b, mw, vw, mb, vb = snap[1 + 6 * i : 7 + 6 * i]
            for dst, src in ((L.w, w), (L.b, b), (L.mw, mw), (L.vw, vw), (L.mb, mb), (L.vb, vb)):
                dst.copy_(src)
            L.wb.copy_(L.w.to(torch.bfloat16))
            L.wt.copy_(L.w.T.to(torch.bfloat16))

    def fit(self, data: RNODataset, epochs: int, graph: bool = True, log=None, lr_schedule=None,
            input_noise: float = 0.0) -> list[float]:  # fmt: skip
        """Train on ``data`` (device-resident); returns the mean loss per epoch.
        ``lr_schedule(epoch)``, when given, sets the step size of each epoch.  ``input_noise``
        adds N(0, input_noise^2) to the normalised strain and rate inputs of every window
        (targets unchanged): the network is taught to be insensitive to input perturbations
        of that size, which keeps its response smooth where a macro solver drives it."""
        c = self.config
        P, T = data.paths, data.steps
        rates = data.rates()
        s = self.scales
        strain_n = (data.strain[:, 1:] / s.strain).float()
        rate_n = (rates / s.rate).float()
        stress_n = (data.stress[:, 1:] / s.stress).float()
        coef = (data.dt / c.tau_ref).float()
        B = min(c.batch_paths, P)
        W = min(c.tbptt_steps, T)
        if T % W != 0:
            raise ValueError("the path length must be a multiple of the truncation window")
        gen = torch.Generator(device="cpu").manual_seed(c.seed)
        noise_gen = torch.Generator(device=self.device).manual_seed(c.seed + 1)
        history = []
        lr_scale = 1.0
        good = self._snapshot()  # start of the last epoch whose loss came out finite
        for epoch in range(epochs):
            base = lr_schedule(epoch) if lr_schedule is not None else c.learning_rate
            self.set_learning_rate(lr_scale * base)
            epoch_start = self._snapshot()
            perm = torch.randperm(P, generator=gen)
            loss_sum = torch.zeros((), dtype=torch.float64, device=self.device)
            windows = 0
            for start in range(0, P - B + 1, B):
                idx = perm[start : start + B].to(self.device)
                z0 = torch.zeros((B, 6), dtype=torch.float32, device=self.device)
                for t0 in range(0, T, W):
                    sl = slice(t0, t0 + W)
                    xs, xr = strain_n[idx, sl].transpose(0, 1), rate_n[idx, sl].transpose(0, 1)
                    if input_noise > 0.0:
                        xs = xs + input_noise * torch.randn(xs.shape, device=xs.device, generator=noise_gen)
                        xr = xr + input_noise * torch.randn(xr.shape, device=xr.device, generator=noise_gen)
                    self.load_window(xs, xr, stress_n[idx, sl].transpose(0, 1), coef[idx, sl].transpose(0, 1), z0)
                    if graph:
                        self._replay(W, B)
                    else:
                        self.window_step(W, B)
                    loss_sum += self._window["loss_part"].sum()  # stays on the device
                    windows += 1
                    z0 = self._window["z"][W].clone()
            history.append(float(loss_sum.item()) / float(windows * B * W * 6))
            if math.isfinite(history[-1]):
                good = epoch_start  # every forward pass of this epoch stayed finite
            else:
                # divergence guard: back to the start of the last finite epoch, half the step
                self._restore(good)
                lr_scale *= 0.5
                self.divergences += 1
                if self.divergences > 8:
                    raise RuntimeError("surrogate training diverged repeatedly (non-finite loss)")
            if log is not None:
                log(epoch, history[-1])
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core GEMM wait timed out during training")
        return history

    def _replay(self, T: int, B: int) -> None:
        w = self._buffers(T, B)
        if self._graph is None:
            # warm up outside capture (first-launch attribute setting), then capture
            stream = torch.cuda.Stream()
            stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(stream):
                self._forward(w, True)
            torch.cuda.current_stream().wait_stream(stream)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._forward(w, True)
                self._backward(w)
                self._adam()
            self._graph = g
        self._graph.replay()

    # -- inference ---------------------------------------------------------------------
    def set_elastic_skip(self, stiffness) -> None:
        """Add K (strain - z) to the stress output, K the given 6x6 stiffness (physical
        units, e.g. the RVE's effective elastic tangent) in normalised units: the network then
        learns the departure from the elastic response with the latent state in strain
        units.  ``None`` removes it."""
        if stiffness is None:
            self.skip = None
        else:
            if not self.fused:
                raise ValueError("the elastic skip term needs the fused kernels (hidden width 128)")
            k = torch.as_tensor(np.asarray(stiffness, dtype=np.float64) * self.scales.strain / self.scales.stress,
                                dtype=torch.float32)  # fmt: skip
            self.skip = k.reshape(6, 6).contiguous().to(self.device)
        self._structs = {}
        self._graph = None

    def predict(self, strain: torch.Tensor, rate: torch.Tensor, z: torch.Tensor, coef: torch.Tensor,
                buffers: dict | None = None) -> tuple[torch.Tensor, torch.Tensor, dict]:  # fmt: skip
        """One step for M points (physical strain (M, 6), rate (M, 6), latent (M, 6), coef
        (M,)): returns (stress (M, 6) in physical units, next latent (M, 6), buffers)."""
        M = int(strain.shape[0])
        if not self.fused:
            return self._predict_unfused(strain, rate, z, coef, buffers)
        dev = self.device
        if buffers is None or buffers["M"] != M:
            buffers = {"M": M, "z": torch.empty((2, M, 6), dtype=torch.float32, device=dev),
                       "stress": torch.empty((1, M, 6), dtype=torch.float32, device=dev)}  # fmt: skip
        s = self.scales
        sn = (strain / s.strain).float().contiguous()
        rn = (rate / s.rate).float().contiguous()
        cf = coef.float().contiguous()
        buffers["z"][0].copy_(z)
        c = _native.RNOWindowC()
        c.B, c.T, c.hidden = M, 1, self.config.hidden
        c.strain, c.rate, c.coef, c.z = sn.data_ptr(), rn.data_ptr(), cf.data_ptr(), buffers["z"].data_ptr()
        for i, L in enumerate(self.layers):
            c.W[i], c.bias[i] = L.wb.data_ptr(), L.b.data_ptr()
        c.skip = None if self.skip is None else self.skip.data_ptr()
        c.stress = buffers["stress"].data_ptr()
        c.err = self.err.data_ptr()
        _check(self.lib.cib_rno_window_forward(ctypes.byref(c), _native.stream_ptr()), "cib_rno_window_forward")
        return buffers["stress"][0] * s.stress, buffers["z"][1], buffers

    def predict_normalized(self, strain_n: torch.Tensor, rate_n: torch.Tensor, coef: torch.Tensor, z: torch.Tensor,
                           stress_n: torch.Tensor) -> None:  # fmt: skip
        """One fused step on prepared inputs: normalised fp32 strain and rate (M, 6), coef
        (M,), latent buffer z (2, M, 6) with the current latent in z[0] (z[1] receives the
        next), normalised stress out (M, 6).  Fused kernels only (hidden width 128)."""
        if not self.fused:
            raise ValueError("predict_normalized needs the fused kernels (hidden width 128)")
        c = _native.RNOWindowC()
        c.B, c.T, c.hidden = int(strain_n.shape[0]), 1, self.config.hidden
        c.strain, c.rate, c.coef, c.z = strain_n.data_ptr(), rate_n.data_ptr(), coef.data_ptr(), z.data_ptr()
        for i, L in enumerate(self.layers):
            c.W[i], c.bias[i] = L.wb.data_ptr(), L.b.data_ptr()
        c.skip = None if self.skip is None else self.skip.data_ptr()
        c.stress = stress_n.data_ptr()
        c.err = self.err.data_ptr()
        _check(self.lib.cib_rno_window_forward(ctypes.byref(c), _native.stream_ptr()), "cib_rno_window_forward")

    def _predict_unfused(self, strain, rate, z, coef, buffers):
        M = int(strain.shape[0])
        dev, h = self.device, self.config.hidden
        if buffers is None or buffers["M"] != M:
            bf = torch.bfloat16
            buffers = {"M": M, "X": torch.empty((M, IN_PAD), dtype=bf, device=dev),
                       "H": [torch.empty((M, h), dtype=bf, device=dev) for _ in range(2)],
                       "Y": torch.empty((M, OUT_PAD), dtype=torch.float32, device=dev),
                       "zn": torch.empty((M, 6), dtype=torch.float32, device=dev)}  # fmt: skip
        s = self.scales
        sn = (strain / s.strain).float().contiguous()
        rn = (rate / s.rate).float().contiguous()
        zf = z.float().contiguous()
        cf = coef.float().contiguous()
        sp = _native.stream_ptr()
        _check(self.lib.cib_rno_input(M, sn.data_ptr(), rn.data_ptr(), zf.data_ptr(), buffers["X"].data_ptr(), None, 0, 0,
                                      sp), "cib_rno_input")  # fmt: skip
        a = buffers["X"]
        for i in range(3):
            out = buffers["H"][i % 2]
            gemm(EPI_BIAS_GELU, a, self.layers[i].wb, bias=self.layers[i].b, h=out, err=self.err)
            a = out
        gemm(EPI_BIAS_F32, a, self.layers[3].wb, bias=self.layers[3].b, c=buffers["Y"], err=self.err)
        _check(self.lib.cib_rno_forward_tail(M, buffers["Y"].data_ptr(), None, cf.data_ptr(), zf.data_ptr(),
                                             buffers["zn"].data_ptr(), None, 0.0, None, sp), "cib_rno_forward_tail")  # fmt: skip
        stress = buffers["Y"][:, :6] * s.stress
        return stress, buffers["zn"], buffers

    def rollout(self, data: RNODataset) -> torch.Tensor:
        """Stress predictions (P, T, 6) (physical units) along every path of ``data``."""
        P, T = data.paths, data.steps
        rates = data.rates()
        if self.fused and P > 0:
            s = self.scales
            dev = self.device
            sn = (data.strain[:, 1:] / s.strain).float().transpose(0, 1).contiguous()
            rn = (rates / s.rate).float().transpose(0, 1).contiguous()
            cf = (data.dt / self.config.tau_ref).float().transpose(0, 1).contiguous()
            zs = torch.zeros((T + 1, P, 6), dtype=torch.float32, device=dev)
            st = torch.empty((T, P, 6), dtype=torch.float32, device=dev)
            c = _native.RNOWindowC()
            c.B, c.T, c.hidden = P, T, self.config.hidden
            c.strain, c.rate, c.coef, c.z = sn.data_ptr(), rn.data_ptr(), cf.data_ptr(), zs.data_ptr()
            for i, L in enumerate(self.layers):
                c.W[i], c.bias[i] = L.wb.data_ptr(), L.b.data_ptr()
            c.skip = None if self.skip is None else self.skip.data_ptr()
            c.stress = st.data_ptr()
            c.err = self.err.data_ptr()
            _check(self.lib.cib_rno_window_forward(ctypes.byref(c), _native.stream_ptr()), "cib_rno_window_forward")
            return (st * s.stress).transpose(0, 1).contiguous()
        z = torch.zeros((P, 6), dtype=torch.float32, device=self.device)
        out = torch.empty((P, T, 6), dtype=torch.float32, device=self.device)
        buf = None
        for t in range(T):
            stress, zn, buf = self.predict(data.strain[:, t + 1], rates[:, t], z, data.dt[:, t] / self.config.tau_ref, buf)
            out[:, t] = stress
            z = zn.clone()
        return out
