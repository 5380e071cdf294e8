"""Differentiable conjugate-pair FFTs for PyTorch: the FP64 and double-double tiers.

The transform y = F x is linear, so its vector-Jacobian product is the
adjoint: for a real loss L of (Re y, Im y) with cotangent g = dL/dRe y +
i dL/dIm y, the cotangent of x is F^H g = conj(F conj(g)) = N F^-1 g, which the
library computes on the device as the unscaled inverse (its first launch reads
the real and imaginary planes exchanged and its last writes them exchanged).
No intermediate is saved: the backward pass needs only the plan.

Tensors use the library's device layouts.  FP64: float64 CUDA tensors of
shape (2, B, n), all real parts (signal after signal), then all imaginary
parts.  Double-double: shape (2, 2, B, n), [re, im] x [hi, lo].

Double-double cotangents are double-double numbers too: the gradient handed
to the backward pass for y is read as hi + lo per component (the value of
dL/dy to about 2^-104 relative), and the gradient returned for x is dL/dx as a
(hi, lo) pair, computed by the adjoint transform in double-double arithmetic.
A caller that forms the cotangent in plain float64 (hi only, lo zero) gets a
float64-accurate gradient; one that forms it in double-double gets a
double-double one.
"""
from __future__ import annotations

import torch

from . import DDPlan, DPlan, DPlanND

_plans: dict = {}
_dd_plans: dict = {}


def _plan(dims):
    key = tuple(dims)
    if key not in _plans:
        _plans[key] = DPlan(key[0]) if len(key) == 1 else DPlanND(key)
    return _plans[key]


class ConjugatePairFFT(torch.autograd.Function):
    """y = FFT(x) on planes (2, B, *dims); backward = the adjoint transform."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, dims: tuple, inverse: bool):
        if x.dtype != torch.float64 or not x.is_cuda:
            raise TypeError("expected a float64 CUDA tensor of shape (2, B, *dims)")
        x = x.contiguous()
        batch = x.shape[1]
        plan = _plan(dims)
        y = torch.empty_like(x)
        s = torch.cuda.current_stream().cuda_stream
        plan.execute_device(batch, x.data_ptr(), y.data_ptr(), stream=s, inverse=inverse)
        ctx.dims, ctx.inverse = dims, inverse
        return y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        gy = gy.contiguous()
        gx = torch.empty_like(gy)
        s = torch.cuda.current_stream().cuda_stream
        # the adjoint of the forward transform is the unscaled inverse, and vice versa
        _plan(ctx.dims).execute_device(gy.shape[1], gy.data_ptr(), gx.data_ptr(), stream=s,
                                       inverse=not ctx.inverse)
        return gx, None, None


def fft(z: torch.Tensor, inverse: bool = False, ndim: int = 1) -> torch.Tensor:
    """Differentiable transform of a complex128 CUDA tensor over its last `ndim`
    dimensions (each a power of two); unscaled in both directions."""
    dims = tuple(z.shape[z.dim() - ndim:])
    lead = z.shape[: z.dim() - ndim]
    zz = z.reshape((-1,) + dims)
    planes = torch.stack((zz.real, zz.imag)).reshape((2, zz.shape[0], -1))
    y = ConjugatePairFFT.apply(planes, dims, inverse)
    return torch.complex(y[0], y[1]).reshape(lead + dims)


def _dd_plan(n: int):
    if n not in _dd_plans:
        _dd_plans[n] = DDPlan(n)
    return _dd_plans[n]


class DDConjugatePairFFT(torch.autograd.Function):
    """Double-double y = FFT(x) on planes (2, 2, B, n) = [re, im] x [hi, lo];
    backward = the adjoint in double-double (the unscaled inverse on the
    device: planes exchanged in the first and the last launch)."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, inverse: bool):
        if x.dtype != torch.float64 or not x.is_cuda or x.dim() != 4 or x.shape[:2] != (2, 2):
            raise TypeError("expected a float64 CUDA tensor of shape (2, 2, B, n)")
        x = x.contiguous()
        batch, n = x.shape[2], x.shape[3]
        y = torch.empty_like(x)
        s = torch.cuda.current_stream().cuda_stream
        _dd_plan(n).execute_device(batch, x.data_ptr(), y.data_ptr(), stream=s, inverse=inverse)
        ctx.inverse = inverse
        return y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        gy = gy.contiguous()
        gx = torch.empty_like(gy)
        s = torch.cuda.current_stream().cuda_stream
        _dd_plan(gy.shape[3]).execute_device(gy.shape[2], gy.data_ptr(), gx.data_ptr(), stream=s,
                                             inverse=not ctx.inverse)
        return gx, None


def dd_fft(x: torch.Tensor, inverse: bool = False) -> torch.Tensor:
    """Differentiable double-double transform of planes (2, 2, B, n) = [re, im]
    x [hi, lo] (n a power of two), unscaled in both directions."""
    return DDConjugatePairFFT.apply(x, inverse)
