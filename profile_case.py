"""Run the device-resident multiprecision transform on synthetic limb planes.

A small, self-contained driver for profilers (ncu) and quick timing:

    python profile_case.py --n 1024 --prec 1024 --batch 512 --reps 2

The input planes are random two's-complement fixed-point values of magnitude
below 2^F (F = the plan's fraction bits), i.e. a block-normalised signal with
components in (-1, 1): exactly what packing uniform [-1,1) mpfr_t inputs
produces.  Prints per-launch milliseconds of the last repetition.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from mpfft_b200.mparray import synthetic_planes  # noqa: E402


def run_fp64(a) -> None:
    """FP64 tier: batch of signals in the device layout [c][b][p]; reports
    time per transform batch and in+out bytes / time."""
    import torch

    import mpfft_b200 as M

    plan = M.DPlan(a.n)
    g = torch.Generator(device="cuda").manual_seed(1)
    d_in = torch.rand((2, a.batch, a.n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    d_out = torch.empty_like(d_in)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), stream=s.cuda_stream)
    e0.record(s)
    for _ in range(a.reps):
        plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    nbytes = 2 * d_in.numel() * 8
    print(f"fp64 n={a.n} batch={a.batch}: {ms:.4f} ms per batch, {a.batch / ms * 1e3:.0f} FFT/s, "
          f"in+out {nbytes / ms / 1e6:.0f} GB/s")


def run_dd(a) -> None:
    """Double-double tier: layout [c][h][b][p]; time per batch and in+out bytes / time."""
    import torch

    import mpfft_b200 as M

    plan = M.DDPlan(a.n)
    g = torch.Generator(device="cuda").manual_seed(1)
    hi = torch.rand((2, a.batch, a.n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    d_in = torch.stack((hi[0], hi[0] * 2.0 ** -60, hi[1], hi[1] * 2.0 ** -60)).contiguous()
    d_out = torch.empty_like(d_in)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), stream=s.cuda_stream)
    e0.record(s)
    for _ in range(a.reps):
        plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    nbytes = 2 * d_in.numel() * 8
    print(f"dd n={a.n} batch={a.batch}: {ms:.4f} ms per batch, {a.batch / ms * 1e3:.0f} FFT/s, "
          f"in+out {nbytes / ms / 1e6:.0f} GB/s")


def main():
    import torch

    import mpfft_b200 as M

    ap = argparse.ArgumentParser()
    ap.add_argument("--tier", default="mp", choices=["mp", "fp64", "dd"])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--prec", type=int, default=1024)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--no-tensor", action="store_true", help="large precision: integer-pipe products")
    ap.add_argument("--force-tensor", action="store_true", help="tensor-core products from 8 limbs up")
    ap.add_argument("--row-products", action="store_true", help="batched limb levels: row-by-row products")
    a = ap.parse_args()
    if a.tier == "fp64":
        run_fp64(a)
        return
    if a.tier == "dd":
        run_dd(a)
        return
    plan = M.MpPlan(a.n, a.prec, tensor="force" if a.force_tensor else not a.no_tensor, row_products=a.row_products)
    host = synthetic_planes(a.n, plan.limbs, plan.frac_bits, a.batch)
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    s = torch.cuda.current_stream().cuda_stream
    ms = None
    for _ in range(a.reps):
        ms = plan.execute_device_timed(a.batch, d_in.data_ptr(), d_out.data_ptr(), s)
    torch.cuda.synchronize()
    sched = plan.schedule()
    print(f"n={a.n} prec={a.prec} limbs={plan.limbs} batch={a.batch} total={sum(ms):.3f} ms "
          f"({a.batch / sum(ms) * 1e3:.0f} FFT/s)")
    print("leaf", round(ms[0], 4), " ".join(f"n{nn}:{t:.4f}" for (nn, _), t in zip(sched, ms[1:])))


if __name__ == "__main__":
    main()
