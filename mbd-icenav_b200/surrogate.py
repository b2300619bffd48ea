"""The learned screening surrogate: a conv + MLP network trained with BF16
tensor-core kernels (fp32 accumulation, Adam on fp32 master weights).

No counterpart in the reference.  The reference's MBD planner scores every
sample of its population with ``jax.vmap(cost_fn)`` inside the reverse
diffusion step (``jax_mbd_planner.py:1363-1380``); ``planner.py`` replaces
that batch by this network's prediction of the DEM's ice terms, and re-scores
the best few samples with the plain batched DEM.

Network (per sample):
  costmap patch (64 x 64, 1 channel, NHWC)
    -> 4 x [3x3 convolution, stride 2, padding 1, ReLU]: 32, 64, 128, 128
       channels (64 -> 32 -> 16 -> 8 -> 4 pixels), as im2col + GEMM
    -> flatten 4 x 4 x 128 = 2048
  [2048 | ship state (6) | controls (H x 2) | log1p of the costmap value at
  each pose of the candidate's rigid-ship path (H) | log1p of what that path
  sweeps through the ice window (8: elements hit, their mass, kinetic-energy
  and momentum proxies, bonds cut)] zero-padded to a multiple of 64
    -> 3 x [fully connected 512, ReLU] -> fully connected 3
  outputs: the standardised log1p transforms of (ice kinetic energy
  transferred, hull impulse, bonds broken).

Every multiply is ``sg_gemm`` (tcgen05.mma, bf16 in, fp32 accumulate); the
rest is the glue kernels of ``surrogate_b200.h``.  Torch tensors only hold
device memory (and draw the initial weights).

FLOPs per sample (forward): conv 2 * (32*32*32*64 + 16*16*64*320 + 8*8*128*576
+ 4*4*128*1152) with padded K, MLP 2 * (in*512 + 2*512*512 + 512*3).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import sg_ops as ops

_torch = None


def _tm():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


PATCH = 64
CONV = ((1, 32), (32, 64), (64, 128), (128, 128))  # (C_in, C_out) per layer
HIDDEN = 512
N_OUT = 3
OUT_ROWS = 64  # stored rows of the output layer (N_OUT live)
N_SHIP = 6
N_STEP = 3  # per-step inputs: normalised surge and yaw controls, the path's costmap value
N_SWEEP = 8  # what the rigid-ship path sweeps through the ice window (dem_rollout_sweep_features)


def kpad_of(c_in: int) -> int:
    return ((9 * c_in + 63) // 64) * 64


def enc_dim() -> int:
    s = PATCH >> len(CONV)
    return s * s * CONV[-1][1]


def x_dim(horizon: int) -> int:
    return ((enc_dim() + N_SHIP + N_STEP * horizon + N_SWEEP + 63) // 64) * 64


def flops_per_sample(horizon: int) -> dict:
    """Forward FLOPs of one sample (padded operand sizes, as the GEMMs run them)."""
    conv, s = 0, PATCH
    for cin, cout in CONV:
        s //= 2
        conv += 2 * s * s * cout * kpad_of(cin)
    xd = x_dim(horizon)
    mlp = 2 * (xd * HIDDEN + 2 * HIDDEN * HIDDEN + HIDDEN * OUT_ROWS)
    return {"encoder": conv, "mlp": mlp}


@dataclass
class Param:
    """One weight matrix (rows = outputs, cols = inputs) and its bias."""
    p: object       # fp32 master weights (rows, cols)
    w: object       # bf16 copy (rows, cols): the GEMM's B operand in the forward pass
    wt: object      # bf16 transpose (cols, rows): B operand of the input-gradient GEMM
    b: object       # fp32 bias (rows,)
    g: object       # fp32 weight gradient
    gb: object      # fp32 bias gradient
    m: object
    v: object
    mb: object
    vb: object
    bw: object      # bf16 scratch written by the bias's Adam step
    fan_in: int


class SurrogateNet:
    """Weights, Adam state and the forward / backward passes."""

    def __init__(self, horizon: int = 64, device="cuda", seed: int = 0):
        torch = _tm()
        self.device = torch.device(device)
        self.horizon = int(horizon)
        self.xdim = x_dim(horizon)
        self.n_extra = N_SHIP + N_STEP * self.horizon + N_SWEEP
        gen = torch.Generator().manual_seed(seed)
        self.conv: List[Param] = []
        for cin, cout in CONV:
            kp = kpad_of(cin)
            self.conv.append(self._param(cout, kp, 9 * cin, gen))
        # the output layer is stored with OUT_ROWS rows, of which the first N_OUT
        # are live (the rest stay zero: their gradients are zero), so that every
        # operand keeps a row stride that is a multiple of 8
        dims = [self.xdim, HIDDEN, HIDDEN, HIDDEN, OUT_ROWS]
        self.fc: List[Param] = [self._param(dims[i + 1], dims[i], dims[i], gen, live=N_OUT if i == 3 else None)
                                for i in range(4)]
        self.t = 0
        self._bufs = {}

    def _param(self, rows, cols, fan_in, gen, live=None) -> Param:
        torch = _tm()
        dev = self.device
        live = rows if live is None else live
        p = torch.zeros((rows, cols), dtype=torch.float32)
        p[:live, :fan_in] = torch.randn((live, fan_in), generator=gen) * math.sqrt(2.0 / fan_in)
        p = p.to(dev)
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)
        w = ops.to_bf16(p)
        wt = ops.transpose(w)
        return Param(p=p, w=w, wt=wt, b=z(rows), g=z(rows, cols), gb=z(rows), m=z(rows, cols), v=z(rows, cols),
                     mb=z(rows), vb=z(rows), bw=torch.zeros((1, rows), dtype=torch.bfloat16, device=dev),
                     fan_in=fan_in)

    def params(self) -> List[Param]:
        return self.conv + self.fc

    _STATE = ("p", "w", "wt", "b", "m", "v", "mb", "vb", "bw")

    def state(self):
        """A device copy of the weights and the Adam state (``load_state`` puts it back)."""
        return [tuple(getattr(q, k).clone() for k in self._STATE) for q in self.params()], self.t

    def load_state(self, st):
        tensors, t = st
        for q, xs in zip(self.params(), tensors):
            for k, x in zip(self._STATE, xs):
                getattr(q, k).copy_(x)
        self.t = t

    def n_params(self) -> int:
        return sum(int(p.fan_in * p.p.shape[0] + p.p.shape[0]) for p in self.params())

    # ── buffers ─────────────────────────────────────────────────────────────
    def _buf(self, name, shape, dtype):
        torch = _tm()
        t = self._bufs.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t

    # ── forward ─────────────────────────────────────────────────────────────
    def encode(self, patches, tag: str = "enc"):
        """patches (P, 64, 64, 1) bf16 -> encoder activations (P, 2048) bf16;
        keeps every layer's patches and activations for ``backward``."""
        torch = _tm()
        x = patches
        P = int(patches.shape[0])
        acts, cols = [x], []
        s = PATCH
        for li, (layer, (cin, cout)) in enumerate(zip(self.conv, CONV)):
            kp = kpad_of(cin)
            s //= 2
            c = ops.im2col(x, kp, out=self._buf(f"{tag}_cols{li}", (P * s * s, kp), torch.bfloat16))
            y = self._buf(f"{tag}_act{li}", (P * s * s, cout), torch.bfloat16)
            ops.gemm(c, layer.w, out=y, bias=layer.b, relu=True)
            x = y.view(P, s, s, cout)
            acts.append(x)
            cols.append(c)
        self._enc_cache = (acts, cols)
        return x.reshape(P, enc_dim())

    def head(self, enc, extra, enc_row=None, tag: str = "head", keep: bool = False):
        """MLP on rows [enc[enc_row[r]] | extra[r]] -> (R, OUT_ROWS) fp32 (first N_OUT columns live)."""
        torch = _tm()
        R = int(extra.shape[0])
        x = ops.pack_rows(enc, extra, self._buf(f"{tag}_x", (R, self.xdim), torch.bfloat16), enc_row=enc_row)
        hs = [x]
        h = x
        for li, layer in enumerate(self.fc[:-1]):
            y = self._buf(f"{tag}_h{li}", (R, HIDDEN), torch.bfloat16)
            ops.gemm(h, layer.w, out=y, bias=layer.b, relu=True)
            hs.append(y)
            h = y
        out = self._buf(f"{tag}_out", (R, OUT_ROWS), torch.float32)
        ops.gemm(h, self.fc[-1].w, out=out, bias=self.fc[-1].b)
        if keep:
            self._head_cache = hs
        return out

    def forward(self, patches, extra, keep: bool = False):
        enc = self.encode(patches)
        return self.head(enc, extra, keep=keep)

    # ── backward ────────────────────────────────────────────────────────────
    def _weight_grad(self, layer: Param, dy, x, tag):
        """layer.g = dy^T x, layer.gb = column sums of dy (dy (M, N) bf16, x (M, K) bf16)."""
        torch = _tm()
        M, N = dy.shape
        K = x.shape[1]
        dyt = ops.transpose(dy, out=self._buf(f"{tag}_dyt", (N, M), torch.bfloat16))
        xt = ops.transpose(x, out=self._buf(f"{tag}_xt", (K, M), torch.bfloat16))
        ops.gemm(dyt, xt, out=layer.g)
        ops.colsum(dy, out=layer.gb)

    def backward(self, dout):
        """dout (R, OUT_ROWS) bf16: gradient of the loss at the head's output
        (zero beyond the first N_OUT columns).  Fills every layer's g / gb."""
        torch = _tm()
        hs = self._head_cache
        acts, cols = self._enc_cache
        R = int(dout.shape[0])
        d = dout
        for li in range(len(self.fc) - 1, -1, -1):
            layer = self.fc[li]
            x = hs[li]
            self._weight_grad(layer, d, x, f"fc{li}")
            if li > 0:
                dx = self._buf(f"fc{li}_dx", (R, x.shape[1]), torch.bfloat16)
                ops.gemm(d, layer.wt, out=dx, mask=x)  # times the ReLU derivative of the layer below
                d = dx
            else:
                # into the encoder: the first enc_dim input columns come from it
                E = enc_dim()
                enc_act = acts[-1].reshape(-1, E)
                if enc_act.shape[0] != R:
                    raise ValueError("backward needs one encoder row per head row (training batches)")
                denc = self._buf("fc0_denc", (R, E), torch.bfloat16)
                ops.gemm(d, layer.wt[:E], out=denc, mask=enc_act)
                d = denc
        # encoder: d is dY of the last conv layer, (R * 4 * 4, 128) in NHWC order
        s = PATCH >> len(CONV)
        P = R
        for li in range(len(self.conv) - 1, -1, -1):
            layer = self.conv[li]
            cin, cout = CONV[li]
            kp = kpad_of(cin)
            dy = d.reshape(P * s * s, cout)
            self._weight_grad(layer, dy, cols[li], f"conv{li}")
            if li > 0:
                dcols = self._buf(f"conv{li}_dcols", (P * s * s, kp), torch.float32)
                ops.gemm(dy, layer.wt, out=dcols)
                H = 2 * s
                d = ops.col2im(dcols, (P, H, H, cin), kp, act=acts[li],
                               out=self._buf(f"conv{li}_dx", (P, H, H, cin), torch.bfloat16))
                d = d.reshape(P * H * H, cin)
            s *= 2

    def adam_step(self, lr: float):
        self.t += 1
        for layer in self.params():
            ops.adam(layer.p, layer.g, layer.m, layer.v, lr, self.t, layer.w, layer.wt)
            ops.adam(layer.b.view(1, -1), layer.gb.view(1, -1), layer.mb.view(1, -1), layer.vb.view(1, -1), lr,
                     self.t, layer.bw)
