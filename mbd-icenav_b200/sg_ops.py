"""Tensor wrappers of the surrogate's device kernels (``include/surrogate_b200.h``).

PyTorch tensors are device buffers here: every op below hands their pointers
to ``libdem_b200.so`` and launches on torch's current stream; no torch
compute kernel runs on these paths.  bf16 tensors are ``torch.bfloat16``.
"""
from __future__ import annotations

import ctypes as C

from . import _abi

_torch = None


def _tm():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def lib():
    return _abi.load_library()


def _p(t):
    return None if t is None else C.c_void_p(int(t.data_ptr()))


def _stream(t):
    return C.c_void_p(_tm().cuda.current_stream(t.device).cuda_stream)


def _check(rc, name):
    if rc != _abi.SG_OK:
        raise RuntimeError(f"{name} failed with status {rc}")


class ErrorFlag:
    """One device int32 that the GEMM sets when a wait ran out of time."""

    def __init__(self, device):
        self.t = _tm().zeros(1, dtype=_tm().int32, device=device)

    def check(self):
        if int(self.t.item()) != 0:
            raise RuntimeError("a surrogate GEMM wait ran past its time limit")


_flags = {}


def _err(device):
    key = (device.type, device.index)
    if key not in _flags:
        _flags[key] = ErrorFlag(device)
    return _flags[key]


def error_flag(device) -> ErrorFlag:
    return _err(device)


def gemm(A, B, out=None, bias=None, relu=False, mask=None, out_dtype=None):
    """``act(A @ B.T + bias) * (mask > 0)`` on the tensor cores.  A (M, K) and B
    (N, K) bf16 with unit column stride (row strides multiples of 8); out (M, N)
    fp32 or bf16 (a new tensor of ``out_dtype`` when not given)."""
    torch = _tm()
    M, K = A.shape
    N, K2 = B.shape
    if K2 != K or A.dtype != torch.bfloat16 or B.dtype != torch.bfloat16:
        raise ValueError("gemm: A (M, K) and B (N, K) must be bf16 with the same K")
    if A.stride(1) != 1 or B.stride(1) != 1:
        raise ValueError("gemm: operands need unit column stride")
    if out is None:
        out = torch.empty((M, N), dtype=out_dtype or torch.float32, device=A.device)
    if out.stride(1) != 1 or out.shape[0] != M or out.shape[1] < N:
        raise ValueError("gemm: out must be (M, >= N) with unit column stride")
    dt = _abi.SG_OUT_BF16 if out.dtype == torch.bfloat16 else _abi.SG_OUT_F32
    if bias is not None and bias.dtype != torch.float32:
        raise ValueError("gemm: bias must be fp32")
    if mask is not None and (mask.dtype != torch.bfloat16 or mask.stride(1) != 1):
        raise ValueError("gemm: mask must be bf16 with unit column stride")
    _check(lib().sg_gemm(M, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(out), out.stride(0), dt, _p(bias),
                         1 if relu else 0, _p(mask), mask.stride(0) if mask is not None else 0,
                         _p(_err(A.device).t), _stream(A)), "sg_gemm")
    return out


def im2col(X, kpad, out=None):
    """(B, H, W, C) bf16 NHWC -> (B H/2 W/2, kpad) bf16 patches of a 3x3 stride-2 convolution."""
    torch = _tm()
    B, H, W, Cc = X.shape
    if out is None:
        out = torch.empty((B * (H // 2) * (W // 2), kpad), dtype=torch.bfloat16, device=X.device)
    _check(lib().sg_im2col(B, H, W, Cc, _p(X), kpad, _p(out), _stream(X)), "sg_im2col")
    return out


def col2im(dcols, shape, kpad, act=None, out=None):
    """Adjoint of ``im2col`` (fp32 patch gradients -> bf16 NHWC), times (act > 0)."""
    torch = _tm()
    B, H, W, Cc = shape
    if out is None:
        out = torch.empty((B, H, W, Cc), dtype=torch.bfloat16, device=dcols.device)
    _check(lib().sg_col2im(B, H, W, Cc, _p(dcols), kpad, _p(act), _p(out), _stream(dcols)), "sg_col2im")
    return out


def transpose(X, out=None):
    torch = _tm()
    R, Cc = X.shape
    if out is None:
        out = torch.empty((Cc, R), dtype=torch.bfloat16, device=X.device)
    _check(lib().sg_transpose(R, Cc, _p(X), X.stride(0), _p(out), out.stride(0), _stream(X)), "sg_transpose")
    return out


def colsum(X, out=None):
    torch = _tm()
    R, Cc = X.shape
    if out is None:
        out = torch.empty(Cc, dtype=torch.float32, device=X.device)
    _check(lib().sg_colsum(R, Cc, _p(X), X.stride(0), 1 if X.dtype == torch.bfloat16 else 0, _p(out), _stream(X)),
           "sg_colsum")
    return out


def adam(p, g, m, v, lr, t, w, wt=None, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step on fp32 master weights p (rows, cols); refreshes the bf16 copy w (and wt = w.T)."""
    R, Cc = p.shape
    _check(lib().sg_adam(R, Cc, _p(p), _p(g), _p(m), _p(v), float(lr), float(beta1), float(beta2), float(eps), int(t),
                         _p(w), w.stride(0), _p(wt), wt.stride(0) if wt is not None else 0, _stream(p)), "sg_adam")


def mse(pred, target, n_out, grad, loss):
    """Mean squared error over the first n_out columns; grad (rows, ldg) bf16, loss (1,) fp32."""
    R = pred.shape[0]
    _check(lib().sg_mse(R, n_out, _p(pred), pred.stride(0), _p(target), target.stride(0), _p(grad), grad.stride(0),
                        _p(loss), _stream(pred)), "sg_mse")


def pack_rows(enc, extra, x, enc_row=None):
    """MLP input rows: [enc (row enc_row[r], or r) | extra | zeros]."""
    R = x.shape[0]
    enc_dim = 0 if enc is None else enc.shape[1]
    n_extra = 0 if extra is None else extra.shape[1]
    _check(lib().sg_pack_rows(R, enc_dim, _p(enc), enc.stride(0) if enc is not None else 0, _p(enc_row), n_extra,
                              _p(extra), extra.stride(0) if extra is not None else 0, _p(x), x.stride(0), _stream(x)),
           "sg_pack_rows")
    return x


def unpack_grad(dx, enc_dim, act, out):
    R = dx.shape[0]
    _check(lib().sg_unpack_grad(R, enc_dim, _p(dx), dx.stride(0), _p(act), _p(out), _stream(dx)), "sg_unpack_grad")
    return out


def to_bf16(x, out=None):
    torch = _tm()
    if out is None:
        out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    _check(lib().sg_to_bf16(x.numel(), _p(x), _p(out), _stream(x)), "sg_to_bf16")
    return out


def gather_rows(src, idx, out):
    """out[r] = src[idx[r]] for row-major tensors of any dtype (unit inner stride)."""
    es = src.element_size()
    row_bytes = out.shape[1] * es if out.dim() == 2 else out[0].numel() * es
    ld_in = src.stride(0) * es
    ld_out = out.stride(0) * es
    _check(lib().sg_gather_rows(out.shape[0], row_bytes, _p(src), ld_in, _p(idx), _p(out), ld_out, _stream(src)),
           "sg_gather_rows")
    return out
