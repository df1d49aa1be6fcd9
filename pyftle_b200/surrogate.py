"""Learned flow-map surrogate: a Fourier-feature SiLU MLP that predicts the
displacement x(t0 + T) - x0 of a seed over a fixed T, trained on RK4
trajectories from the engine's own window kernels and run by its own BF16
tensor-core kernels (``ftle_mlp_*``; forward, backward and Adam all on the GPU).

The surrogate replaces advection for sliding windows of a fixed length T.  Its
FTLE comes from the network's own flow-map Jacobian (forward-mode tangents of
the features through every layer, one extra pass per input direction), not
from finite differences of BF16 outputs at offset 5e-4, which BF16 rounding
would swamp.  Plain RK4 stays the judge and the fallback: on every field a
sampled fraction of seeds per region is advected with RK4 (neighbour groups at
offset delta, the reference's FTLE, ftle_solver.py:151-161) and every region
whose sampled error exceeds the tolerance is re-advected with RK4.

No counterpart in the reference; it stands where the advection loop of
``FTLESolver.run`` (ftle_solver.py:116-149) stands.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from pyftle_b200 import _lib
from pyftle_b200._device import ptr, require_cuda, stream_ptr


def fourier_frequencies(num: int = 32, *, length: float = 2.0 * math.pi,
                        space_sigma: float = 6.0, time_sigma: float = 0.3,
                        seed: int = 0, dim: int = 2) -> np.ndarray:
    """Frequency rows: 2D (num, 4) float32 (kx, ky, kt, phase); 3D (num, 8) float32
    (kx, ky, kz, kt, phase, 0, 0, 0).  Integer wavenumbers on the periodic box
    [0, length)^dim (the features stay periodic), Gaussian time frequencies.  The
    first rows are pure spatial unit modes, so the lowest harmonics are always present."""
    if dim not in (2, 3):
        raise ValueError("dim must be 2 or 3")
    rng = np.random.default_rng(seed)
    k0 = 2.0 * math.pi / length
    rows = ([(1, 0), (0, 1), (1, 1), (1, -1)] if dim == 2 else
            [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1), (1, 0, 1)])
    out = np.zeros((num, 4 if dim == 2 else 8), dtype=np.float32)
    for i in range(num):
        if i < len(rows):
            k, kt = rows[i], 0.0
        else:
            while True:
                k = np.round(rng.normal(0.0, space_sigma, dim)).astype(int)
                if np.any(k):
                    break
            kt = rng.normal(0.0, time_sigma)
        out[i, :dim] = np.asarray(k, dtype=np.float64) * k0
        out[i, dim] = kt
    return out


@dataclass
class _Layer:
    fan_in: int
    fan_out: int      # logical outputs
    out_pad: int      # rows stored (multiple of 64 for the output layer)
    w_off: int
    b_off: int


class FlowMapMLP:
    """features(x0, t0) -> [hidden x depth, SiLU] -> displacement / out_scale, in 2D
    (freq rows of 4: points (x, y, t0)) or 3D (freq rows of 8: points (x, y, z, t0))."""

    OUT_PAD = 64

    def __init__(self, freq: np.ndarray, *, hidden: int = 256, depth: int = 4,
                 outs: Optional[int] = None, out_scale: float = 1.0, seed: int = 0,
                 device=None):
        self.device = device or require_cuda()
        freq = np.ascontiguousarray(freq, dtype=np.float32)
        if freq.ndim != 2 or freq.shape[1] not in (4, 8) or (2 * freq.shape[0]) % 64:
            raise ValueError("freq must be (F, 4) (2D) or (F, 8) (3D) with 2F a multiple of 64")
        self.dim = 2 if freq.shape[1] == 4 else 3
        outs = self.dim if outs is None else int(outs)
        if hidden % 64 or hidden > 1024:
            raise ValueError("hidden width must be a multiple of 64, at most 1024")
        self.freq_np = freq
        self.freq = torch.from_numpy(freq).to(self.device)
        self.in_features = 2 * freq.shape[0]
        self.hidden, self.depth, self.outs = hidden, depth, outs
        self.out_scale = float(out_scale)
        dims = [self.in_features] + [hidden] * depth
        self.layers: List[_Layer] = []
        off = 0
        for l in range(depth + 1):
            fin = dims[l]
            fout = hidden if l < depth else outs
            pad = hidden if l < depth else self.OUT_PAD
            w_off, off = off, off + pad * fin
            b_off, off = off, off + pad
            self.layers.append(_Layer(fin, fout, pad, w_off, b_off))
        self.num_params = off
        rng = np.random.default_rng(seed)
        w = np.zeros(off, dtype=np.float32)
        for l, L in enumerate(self.layers):
            std = math.sqrt(2.0 / L.fan_in) if l < depth else 0.1 / math.sqrt(L.fan_in)
            W = np.zeros((L.out_pad, L.fan_in), dtype=np.float32)
            W[:L.fan_out] = rng.normal(0.0, std, (L.fan_out, L.fan_in))
            w[L.w_off:L.w_off + W.size] = W.ravel()
        self.w = torch.from_numpy(w).to(self.device)
        self.wb = self.w.to(torch.bfloat16)
        self.g = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._fused = None
        self._ws: Dict[str, torch.Tensor] = {}
        self._ws_rows = 0

    # ---- parameters ----------------------------------------------------------------
    def weight(self, l: int, bf16: bool = False) -> torch.Tensor:
        L = self.layers[l]
        src = self.wb if bf16 else self.w
        return src[L.w_off:L.w_off + L.out_pad * L.fan_in].view(L.out_pad, L.fan_in)

    def bias(self, l: int) -> torch.Tensor:
        L = self.layers[l]
        return self.w[L.b_off:L.b_off + L.out_pad]

    def grad_weight(self, l: int) -> torch.Tensor:
        L = self.layers[l]
        return self.g[L.w_off:L.w_off + L.out_pad * L.fan_in].view(L.out_pad, L.fan_in)

    def grad_bias(self, l: int) -> torch.Tensor:
        L = self.layers[l]
        return self.g[L.b_off:L.b_off + L.out_pad]

    def numpy_params(self) -> Tuple[List[np.ndarray], List[np.ndarray]]:
        """(weights, biases) as float64 numpy arrays (output layer unpadded)."""
        Ws, bs = [], []
        for l, L in enumerate(self.layers):
            Ws.append(self.weight(l).cpu().numpy().astype(np.float64)[:L.fan_out])
            bs.append(self.bias(l).cpu().numpy().astype(np.float64)[:L.fan_out])
        return Ws, bs

    def state_dict(self) -> Dict[str, np.ndarray]:
        return {"w": self.w.cpu().numpy(), "freq": self.freq_np,
                "meta": np.array([self.hidden, self.depth, self.outs], dtype=np.int64),
                "out_scale": np.array([self.out_scale])}

    @classmethod
    def from_state(cls, state: Dict[str, np.ndarray], device=None) -> "FlowMapMLP":
        hidden, depth, outs = (int(x) for x in state["meta"])
        net = cls(state["freq"], hidden=hidden, depth=depth, outs=outs,
                  out_scale=float(state["out_scale"][0]), device=device)
        net.w.copy_(torch.from_numpy(np.asarray(state["w"], dtype=np.float32)))
        net.wb.copy_(net.w.to(torch.bfloat16))
        net._fused = None
        return net

    # ---- workspace -------------------------------------------------------------------
    def _workspace(self, rows: int) -> Dict[str, torch.Tensor]:
        rows = ((rows + 127) // 128) * 128
        if rows <= self._ws_rows:
            return self._ws
        dev, H, F = self.device, self.hidden, self.in_features
        bf, f32 = torch.bfloat16, torch.float32
        ws = {"feat": torch.empty(rows, F, dtype=bf, device=dev),
              "tx": torch.empty(rows, F, dtype=bf, device=dev),
              "ty": torch.empty(rows, F, dtype=bf, device=dev),
              "tz": torch.empty(rows, F, dtype=bf, device=dev) if self.dim == 3 else None,
              "Y": torch.empty(rows, self.OUT_PAD, dtype=f32, device=dev),
              "dY": torch.empty(rows, self.OUT_PAD, dtype=bf, device=dev),
              "Ga": torch.empty(rows, H, dtype=bf, device=dev),
              "Gb": torch.empty(rows, H, dtype=bf, device=dev),
              "Jx": torch.empty(rows, self.OUT_PAD, dtype=f32, device=dev),
              "Jy": torch.empty(rows, self.OUT_PAD, dtype=f32, device=dev),
              "Jz": (torch.empty(rows, self.OUT_PAD, dtype=f32, device=dev)
                     if self.dim == 3 else None),
              "loss": torch.zeros(1, dtype=f32, device=dev)}
        for l in range(self.depth):
            ws[f"Z{l}"] = torch.empty(rows, H, dtype=f32, device=dev)
            ws[f"H{l}"] = torch.empty(rows, H, dtype=bf, device=dev)
        self._ws, self._ws_rows = ws, rows
        return ws

    # ---- passes ----------------------------------------------------------------------
    def _features(self, points: torch.Tensor, n: int, tangents: bool):
        ws = self._workspace(n)
        t = (lambda k: ws[k] if tangents else None)
        if self.dim == 2:
            _lib.call("ftle_mlp_features", ptr(points), n, ptr(self.freq), self.freq.shape[0],
                      ptr(ws["feat"]), ptr(t("tx")), ptr(t("ty")), stream_ptr())
        else:
            _lib.call("ftle_mlp_features3", ptr(points), n, ptr(self.freq), self.freq.shape[0],
                      ptr(ws["feat"]), ptr(t("tx")), ptr(t("ty")), ptr(t("tz")), stream_ptr())
        return ws

    def _forward(self, ws, n: int):
        s = stream_ptr()
        x, ldx = ws["feat"], self.in_features
        for l, L in enumerate(self.layers):
            W = self.weight(l, bf16=True)
            if l < self.depth:
                _lib.call("ftle_mlp_linear", ptr(x), ldx, ptr(W), L.fan_in, ptr(self.bias(l)), n,
                          L.out_pad, L.fan_in, 1, ptr(ws[f"Z{l}"]), L.out_pad, ptr(ws[f"H{l}"]),
                          L.out_pad, ptr(self.err), s)
                x, ldx = ws[f"H{l}"], L.out_pad
            else:
                _lib.call("ftle_mlp_linear", ptr(x), ldx, ptr(W), L.fan_in, ptr(self.bias(l)), n,
                          L.out_pad, L.fan_in, 0, ptr(ws["Y"]), self.OUT_PAD, ptr(None), 0,
                          ptr(self.err), s)

    def _tangent(self, ws, n: int, seed_key: str, out_key: str):
        s = stream_ptr()
        t, ldt = ws[seed_key], self.in_features
        bufs = (ws["Ga"], ws["Gb"])
        for l, L in enumerate(self.layers):
            W = self.weight(l, bf16=True)
            if l < self.depth:
                out = bufs[l & 1]
                _lib.call("ftle_mlp_gemm_dsilu", ptr(t), ldt, 0, ptr(W), L.fan_in, 0, n,
                          L.out_pad, L.fan_in, ptr(ws[f"Z{l}"]), L.out_pad, ptr(out), L.out_pad,
                          ptr(None), ptr(self.err), s)
                t, ldt = out, L.out_pad
            else:
                _lib.call("ftle_mlp_gemm", ptr(t), ldt, 0, ptr(W), L.fan_in, 0, ptr(ws[out_key]),
                          self.OUT_PAD, n, L.out_pad, L.fan_in, 1, 0, ptr(self.err), s)

    def predict(self, points: torch.Tensor, jacobian: bool = False):
        """points (n, dim+1) float64 CUDA (x0, t0).  Returns the network output Y
        (n, OUT_PAD) FP32 views (displacement / out_scale in columns :outs), and with
        ``jacobian`` the tangents dY/dx (, dY/dy, dY/dz) (views into the workspace;
        valid until the next call)."""
        n = self._check_points(points)
        ws = self._features(points, n, jacobian)
        self._forward(ws, n)
        if not jacobian:
            return ws["Y"][:n]
        keys = (("tx", "Jx"), ("ty", "Jy"), ("tz", "Jz"))[:self.dim]
        for seed, out in keys:
            self._tangent(ws, n, seed, out)
        return (ws["Y"][:n],) + tuple(ws[o][:n] for _, o in keys)

    def ftle(self, points: torch.Tensor, T: float, out: Optional[torch.Tensor] = None,
             chunk: int = 1 << 20) -> torch.Tensor:
        """FTLE (float64) of the surrogate flow map at points (n, dim+1), in chunks."""
        n = self._check_points(points)
        if out is None:
            out = torch.empty(n, dtype=torch.float64, device=points.device)
        for i in range(0, n, chunk):
            j = min(n, i + chunk)
            _, *J = self.predict(points[i:j], jacobian=True)
            name = "ftle_mlp_jacobian_ftle" if self.dim == 2 else "ftle_mlp_jacobian_ftle3"
            _lib.call(name, *(ptr(x) for x in J), self.OUT_PAD, j - i, self.out_scale,
                      float(T), ptr(out[i:j]), stream_ptr())
        return out

    def end_positions(self, points: torch.Tensor, chunk: int = 1 << 20) -> torch.Tensor:
        """x0 + predicted displacement, (n, dim) float64."""
        n = self._check_points(points)
        out = torch.empty(n, self.dim, dtype=torch.float64, device=points.device)
        name = ("ftle_mlp_apply_displacement" if self.dim == 2
                else "ftle_mlp_apply_displacement3")
        for i in range(0, n, chunk):
            j = min(n, i + chunk)
            y = self.predict(points[i:j])
            _lib.call(name, ptr(points[i:j]), ptr(y), self.OUT_PAD, j - i, self.out_scale,
                      ptr(out[i:j]), stream_ptr())
        return out

    def loss_and_grads(self, points: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """Forward + backward on one batch; gradients are ADDED to self.g.

        target: (n, outs) float32, the displacement divided by out_scale.
        Returns the device loss (mean over rows of the squared error)."""
        n = self._check_points(points)
        if target.dtype != torch.float32 or not target.is_contiguous() or \
                tuple(target.shape) != (n, self.outs):
            raise ValueError(f"target must be a contiguous float32 ({n}, {self.outs}) tensor")
        s = stream_ptr()
        ws = self._features(points, n, False)
        self._forward(ws, n)
        ws["loss"].zero_()
        last = self.depth
        _lib.call("ftle_mlp_mse_grad", ptr(ws["Y"]), self.OUT_PAD, ptr(target), self.outs, n,
                  ptr(ws["dY"]), self.OUT_PAD, ptr(self.grad_bias(last)), ptr(ws["loss"]), s)
        g, ldg = ws["dY"], self.OUT_PAD
        bufs = (ws["Ga"], ws["Gb"])
        splits = max(1, min(n // 128 // 8, 74))
        for l in range(last, -1, -1):
            L = self.layers[l]
            x = ws["feat"] if l == 0 else ws[f"H{l - 1}"]
            # dW_l (out_pad x fan_in) += G^T X  (contraction over the batch)
            _lib.call("ftle_mlp_gemm", ptr(g), ldg, 1, ptr(x), L.fan_in, 1,
                      ptr(self.grad_weight(l)), L.fan_in, L.out_pad, L.fan_in, n, splits, 1,
                      ptr(self.err), s)
            if l > 0:
                # dZ_{l-1} = (G W_l) * silu'(Z_{l-1}); bias gradient of layer l-1
                out = bufs[l & 1]
                P = self.layers[l - 1]
                _lib.call("ftle_mlp_gemm_dsilu", ptr(g), ldg, 0, ptr(self.weight(l, bf16=True)),
                          L.fan_in, 1, n, L.fan_in, L.out_pad, ptr(ws[f"Z{l - 1}"]), P.out_pad,
                          ptr(out), P.out_pad, ptr(self.grad_bias(l - 1)), ptr(self.err), s)
                g, ldg = out, P.out_pad
        return ws["loss"]

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
                  weight_decay: float = 0.0):
        self.step += 1
        _lib.call("ftle_mlp_adam", ptr(self.w), ptr(self.g), ptr(self.m), ptr(self.v),
                  ptr(self.wb), self.num_params, float(lr), float(beta1), float(beta2),
                  float(eps), self.step, float(weight_decay), stream_ptr())

    # ---- fused inference ---------------------------------------------------------------
    @property
    def supports_fused(self) -> bool:
        """The fused kernel's fixed shape: 32 frequencies, 4 x 256 hidden, 2 outputs."""
        return (self.dim == 2 and self.in_features == 64 and self.hidden == 256
                and self.depth == 4 and self.outs == 2)

    def _fused_params(self):
        if getattr(self, "_fused_key", None) == (self.step, id(self.w)) and self._fused is not None:
            return self._fused
        if not self.supports_fused:
            raise ValueError("the fused kernel needs 32 frequencies, 4 x 256 hidden, 2 outputs")
        nbytes = int(_lib.load().ftle_surrogate_packed_bytes())
        packed = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        ws = [self.weight(l, bf16=True) for l in range(5)]
        _lib.call("ftle_surrogate_pack", *(ptr(w) for w in ws), ptr(packed), stream_ptr())
        bias = torch.cat([self.bias(l) for l in range(4)] + [self.bias(4)[:16]]).contiguous()
        self._fused = (packed, bias)
        self._fused_key = (self.step, id(self.w))
        return self._fused

    def ftle_fused(self, seeds: torch.Tensor, t0: float, T: float,
                   out: Optional[torch.Tensor] = None,
                   end_positions: Optional[torch.Tensor] = None) -> torch.Tensor:
        """FTLE (float64) of the surrogate flow map at (n, 2) seeds all starting at t0,
        in one launch of the fused tensor-core kernel (optionally also the predicted
        end positions, (n, 2) float64)."""
        if seeds.dtype != torch.float64 or not seeds.is_cuda or not seeds.is_contiguous() \
                or seeds.ndim != 2 or seeds.shape[1] != 2:
            raise ValueError("seeds must be a contiguous (n, 2) float64 CUDA tensor")
        n = seeds.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float64, device=seeds.device)
        packed, bias = self._fused_params()
        _lib.call("ftle_surrogate_ftle", ptr(seeds), n, float(t0), ptr(packed), ptr(bias),
                  ptr(self.freq), self.out_scale, float(T), ptr(out), ptr(end_positions),
                  ptr(self.err), stream_ptr())
        return out

    def check_errors(self):
        if int(self.err.item()) != 0:
            self.err.zero_()
            raise RuntimeError("a tensor-core wait timed out in an MLP kernel")

    def _check_points(self, points: torch.Tensor) -> int:
        d = self.dim + 1
        if points.dtype != torch.float64 or not points.is_cuda or not points.is_contiguous() \
                or points.ndim != 2 or points.shape[1] != d:
            raise ValueError(f"points must be a contiguous (n, {d}) float64 CUDA tensor")
        n = points.shape[0]
        if n % 8:
            raise ValueError("the number of points must be a multiple of 8")
        return n


# ---------------------------------------------------------------------------------------
# training data and training
# ---------------------------------------------------------------------------------------

def rk4_displacements(series, points: torch.Tensor, *, T: float, h: float,
                      snapshot_dt: float, chunk: int = 1 << 22) -> torch.Tensor:
    """Displacement (n, dim) float64 of each (x0, t0) point (n, dim+1) over T by RK4
    through an FP64 series (time-blended; the plain window kernel advects every point
    independently; points with equal t0 share a launch)."""
    from pyftle_b200.window import run_window

    if series.storage != _lib.F64:
        raise ValueError("training trajectories come from an FP64 series")
    dim = series.grid.dim
    steps = int(round(T / h))
    if abs(steps * h - T) > 1e-9 * max(1.0, T):
        raise ValueError("T must be a whole number of steps h")
    t0s = points[:, dim]
    uniq = torch.unique(t0s).cpu().numpy()
    out = torch.empty(points.shape[0], dim, dtype=torch.float64, device=points.device)
    for t0 in uniq:
        idx = torch.nonzero(t0s == float(t0)).squeeze(1)
        for i in range(0, idx.numel(), chunk):
            sel = idx[i:i + chunk]
            m = sel.numel()
            pad = (-m) % (2 * dim)
            p = points[sel, :dim]
            if pad:
                p = torch.cat([p, p[:pad]])
            p = p.contiguous()
            x0 = p.clone()
            run_window(series, p, integrator="rk4", time_mode="blend", h=h, num_steps=steps,
                       t0=float(t0), snapshot_dt=snapshot_dt, with_ftle=False)
            out[sel] = (p - x0)[:m]
    return out


@dataclass
class TrainConfig:
    steps: int = 3000
    batch: int = 65536
    lr: float = 2e-3
    lr_final: float = 2e-5
    warmup: int = 100
    weight_decay: float = 0.0
    log_every: int = 0
    seed: int = 0


def train(net: FlowMapMLP, points: torch.Tensor, displacement: torch.Tensor,
          cfg: TrainConfig = TrainConfig()) -> List[Tuple[int, float]]:
    """Adam with linear warm-up and cosine decay on random batches of the set.
    Returns [(step, loss)] at the log points (every cfg.log_every steps, and the last)."""
    n = points.shape[0]
    B = min(cfg.batch, n - n % 128)
    target = (displacement / net.out_scale).to(torch.float32).contiguous()
    gen = torch.Generator(device=points.device)
    gen.manual_seed(cfg.seed)
    log = []
    acc = torch.zeros(1, dtype=torch.float32, device=points.device)
    since = 0  # steps accumulated in acc
    for it in range(cfg.steps):
        idx = torch.randint(0, n, (B,), device=points.device, generator=gen)
        loss = net.loss_and_grads(points[idx].contiguous(), target[idx].contiguous())
        acc += loss
        since += 1
        if it < cfg.warmup:
            lr = cfg.lr * (it + 1) / cfg.warmup
        else:
            u = (it - cfg.warmup) / max(1, cfg.steps - cfg.warmup)
            lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1.0 + math.cos(math.pi * u))
        net.adam_step(lr, weight_decay=cfg.weight_decay)
        if (cfg.log_every and (it + 1) % cfg.log_every == 0) or it == cfg.steps - 1:
            log.append((it + 1, float(acc.item()) / since))
            acc.zero_()
            since = 0
    net.check_errors()
    return log


def fit_flow_map(series64, *, T: float, h: float, snapshot_dt: float, t0_values,
                 num_samples: int, length: float = 2.0 * math.pi,
                 freq: Optional[np.ndarray] = None, hidden: int = 256, depth: int = 4,
                 cfg: TrainConfig = TrainConfig(),
                 seed: int = 0) -> Tuple[FlowMapMLP, Dict[str, float]]:
    """Train a FlowMapMLP on ``num_samples`` RK4 trajectories of the FP64 series: seeds
    uniform on the periodic box [0, length)^dim, start times drawn from ``t0_values``.
    Returns the network and timings (seconds) of data generation and training."""
    import time

    dev = require_cuda()
    dim = series64.grid.dim
    g = torch.Generator(device=dev).manual_seed(seed)
    pts = torch.rand(num_samples, dim + 1, generator=g, device=dev, dtype=torch.float64)
    pts[:, :dim] *= length
    t0v = torch.as_tensor(np.asarray(t0_values, dtype=np.float64), device=dev)
    pts[:, dim] = t0v[torch.randint(0, t0v.numel(), (num_samples,), generator=g, device=dev)]
    torch.cuda.synchronize()
    a = time.perf_counter()
    disp = rk4_displacements(series64, pts, T=T, h=h, snapshot_dt=snapshot_dt)
    torch.cuda.synchronize()
    b = time.perf_counter()
    if freq is None:
        freq = fourier_frequencies(32, length=length, dim=dim)
    net = FlowMapMLP(freq, hidden=hidden, depth=depth, out_scale=float(disp.abs().max()),
                     seed=seed)
    log = train(net, pts, disp, cfg)
    torch.cuda.synchronize()
    c = time.perf_counter()
    return net, {"data_s": b - a, "train_s": c - b, "final_loss": log[-1][1],
                 "samples": num_samples, "steps": cfg.steps, "batch": cfg.batch,
                 "hidden": hidden, "depth": depth}


# ---------------------------------------------------------------------------------------
# surrogate FTLE with the RK4 judge
# ---------------------------------------------------------------------------------------

@dataclass
class JudgeReport:
    regions: int
    rejected: int
    sampled: int
    readvected_seeds: int
    region_errors: np.ndarray = field(repr=False)

    @property
    def accepted_fraction(self) -> float:
        return 1.0 - self.rejected / max(1, self.regions)


class SurrogateFTLE:
    """FTLE fields of fixed-length windows on a regular seed grid: the surrogate for
    every seed, RK4 on a sampled fraction of seeds per region as the judge, RK4
    re-advection of every region whose sampled error exceeds ``tol``.

    Error of a region = RMS over its sampled seeds of (surrogate - RK4) FTLE,
    divided by the RMS of the RK4 FTLE over all sampled seeds of the field (the
    field-level relative L2 error restricted to the region).
    """

    def __init__(self, net: FlowMapMLP, series, *, nx: int, ny: int, nz: Optional[int] = None,
                 origin=(0.0, 0.0, 0.0), spacing=(1.0, 1.0, 1.0), T: float, h: float,
                 snapshot_dt: float, delta: float = 5e-4, tile: int = 32,
                 sample_fraction: float = 0.01, tol: float = 1e-3,
                 rk4_chunk_steps: Optional[int] = None, seed: int = 0):
        self.net, self.series = net, series
        self.dim = 2 if nz is None else 3
        if net.dim != self.dim or series.grid.dim != self.dim:
            raise ValueError("network, series and seed grid must have the same dimension")
        self.nx, self.ny, self.nz = nx, ny, (nz or 1)
        self.T, self.h = float(T), float(h)
        self.steps = int(round(T / h))
        self.snapshot_dt, self.delta, self.tol = float(snapshot_dt), float(delta), float(tol)
        self.rk4_chunk_steps = rk4_chunk_steps
        dev = net.device
        axes = [origin[a] + spacing[a] * np.arange(m)
                for a, m in enumerate((nx, ny, nz)[:self.dim])]
        # seeds in the reference's meshgrid-"xy" order: 2D j*nx + i, 3D (j*nx + i)*nz + k
        grids = np.meshgrid(*axes)
        self.centroids = torch.from_numpy(np.column_stack([g.ravel() for g in grids])).to(dev)
        n = self.centroids.shape[0]
        if n % 8:
            raise ValueError("the number of seeds must be a multiple of 8")
        self.points = torch.empty(n, self.dim + 1, dtype=torch.float64, device=dev)
        self.points[:, :self.dim] = self.centroids
        # regions: tile^dim blocks of seeds; region id of every seed
        counts_ax = [(m + tile - 1) // tile for m in (nx, ny, nz)[:self.dim]]
        idx = np.meshgrid(*[np.arange(m) // tile for m in (nx, ny, nz)[:self.dim]])
        if self.dim == 2:
            region = (idx[1] * counts_ax[0] + idx[0]).ravel()
        else:
            region = ((idx[1] * counts_ax[0] + idx[0]) * counts_ax[2] + idx[2]).ravel()
        self.num_regions = int(np.prod(counts_ax))
        self.region_of = torch.from_numpy(region).to(dev)
        order = np.argsort(region, kind="stable")
        counts = np.bincount(region, minlength=self.num_regions)
        starts = np.concatenate(([0], np.cumsum(counts)[:-1]))
        self.region_seeds = [torch.from_numpy(order[s:s + c]).to(dev)
                             for s, c in zip(starts, counts)]
        rng = np.random.default_rng(seed)
        sample = []
        for s, c in zip(starts, counts):
            k = max(1, int(math.ceil(sample_fraction * c)))
            sample.append(order[s + rng.choice(c, size=k, replace=False)])
        self.sample_idx = torch.from_numpy(np.concatenate(sample)).to(dev)
        self.sample_region = self.region_of[self.sample_idx]

    def _rk4_ftle(self, seeds: torch.Tensor, t0: float) -> torch.Tensor:
        from pyftle_b200 import flows
        from pyftle_b200.window import run_window

        c = self.centroids[seeds]
        pos = (flows.seeds_2d_device(c, self.delta) if self.dim == 2
               else flows.seeds_3d_device(c, self.delta))
        return run_window(self.series, pos, integrator="rk4", time_mode="blend", h=self.h,
                          num_steps=self.steps, t0=t0, snapshot_dt=self.snapshot_dt,
                          chunk_steps=self.rk4_chunk_steps)

    def surrogate_field(self, t0: float) -> torch.Tensor:
        """The network's FTLE for every seed (no judge)."""
        if self.net.supports_fused:
            return self.net.ftle_fused(self.centroids, t0, self.T)
        self.points[:, self.dim] = t0
        return self.net.ftle(self.points, self.T)

    def evaluate(self, t0: float) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """(surrogate field, RK4 FTLE of the sampled seeds, error of every region)."""
        f = self.surrogate_field(t0)
        ref = self._rk4_ftle(self.sample_idx, t0)
        err = (f[self.sample_idx] - ref) ** 2
        R = self.num_regions
        num = torch.zeros(R, dtype=torch.float64, device=f.device).index_add_(
            0, self.sample_region, err)
        cnt = torch.zeros(R, dtype=torch.float64, device=f.device).index_add_(
            0, self.sample_region, torch.ones_like(err))
        scale = torch.sqrt(torch.mean(ref * ref)).clamp_min(1e-300)
        return f, ref, torch.sqrt(num / cnt.clamp_min(1)) / scale

    def field(self, t0: float, judge: bool = True,
              tol: Optional[float] = None) -> Tuple[torch.Tensor, Optional[JudgeReport]]:
        """FTLE field of the window starting at t0: surrogate where the judge accepts,
        RK4 at the sampled seeds and in every rejected region."""
        if not judge:
            return self.surrogate_field(t0), None
        tol = self.tol if tol is None else float(tol)
        f, ref, region_err = self.evaluate(t0)
        f[self.sample_idx] = ref
        bad = torch.nonzero(region_err > tol).squeeze(1).cpu().numpy()
        readv = 0
        if bad.size == self.num_regions:
            f = self.reference_field(t0)
            readv = self.centroids.shape[0]
        elif bad.size:
            seeds = torch.cat([self.region_seeds[int(r)] for r in bad])
            f[seeds] = self._rk4_ftle(seeds, t0)
            readv = int(seeds.numel())
        rep = JudgeReport(regions=self.num_regions, rejected=int(bad.size),
                          sampled=int(self.sample_idx.numel()), readvected_seeds=readv,
                          region_errors=region_err.cpu().numpy())
        return f, rep

    def run(self, starts: Sequence[float], writer=None):
        """Sliding windows starting at each of ``starts``.  Returns the fields (host
        arrays) and the judge reports, or writes ``ftle_<t0>`` files with ``writer``."""
        fields, reports = [], []
        for t0 in starts:
            f, rep = self.field(float(t0))
            reports.append(rep)
            arr = f.cpu().numpy()
            if writer is not None:
                writer.write(f"ftle_{float(t0):06f}", arr, self.centroids.cpu().numpy())
            else:
                fields.append(arr)
        return (None if writer is not None else fields), reports

    def reference_field(self, t0: float) -> torch.Tensor:
        """RK4 FTLE of every seed (the method without the surrogate)."""
        all_idx = torch.arange(self.centroids.shape[0], device=self.centroids.device)
        return self._rk4_ftle(all_idx, t0)
