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


def run_multiword(a) -> None:
    """Quad-double or float-float tier: layout [c][h][b][p]; time per batch."""
    import torch

    import mpfft_b200 as M

    plan = M.MultiwordPlan(a.n, a.tier)
    dt = torch.float32 if plan.word_bytes == 4 else torch.float64
    x = (torch.rand((2, plan.words, a.batch, a.n), dtype=torch.float64, device="cuda") * 2 - 1).to(dt)
    x[:, 1:] *= 2.0 ** -60 if dt == torch.float64 else 2.0 ** -30
    y = torch.empty_like(x)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        plan.execute_device(a.batch, x.data_ptr(), y.data_ptr(), stream=s.cuda_stream)
    e0.record(s)
    for _ in range(a.reps):
        plan.execute_device(a.batch, x.data_ptr(), y.data_ptr(), stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    print(f"{a.tier} n={a.n} batch={a.batch}: {ms:.4f} ms per batch, {a.batch / ms * 1e3:.0f} FFT/s")


def run_queue(a) -> None:
    """Uneven batch through the work-queue graph: a.batch signals, N = 2^4 ..
    2^a.lg_max log-uniform, P from {24, 53, 106, 212, 512, 1024}, native tiers."""
    import torch

    import mpfft_b200 as M
    from bench import SEED, fill_uneven_arena

    rng = np.random.default_rng(SEED)
    ns = [1 << int(v) for v in rng.integers(4, a.lg_max + 1, a.batch)]
    ps = [int(v) for v in rng.choice([24, 53, 106, 212, 512, 1024], a.batch)]
    bp = M.BatchPlan(ns, ps, float_tiers="native")
    fill_uneven_arena(M, bp, ns, rng)
    s = torch.cuda.current_stream().cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        bp.execute_device(s)
    e0.record()
    for _ in range(a.reps):
        bp.execute_device(s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    print(f"queue signals={a.batch} lg_max={a.lg_max}: {ms:.3f} ms per graph launch")


def main():
    import torch

    import mpfft_b200 as M

    ap = argparse.ArgumentParser()
    ap.add_argument("--tier", default="mp", choices=["mp", "fp64", "dd", "qd", "ff", "queue"])
    ap.add_argument("--lg-max", type=int, default=12, help="queue: largest log2 N")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--prec", type=int, default=1024)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--no-tensor", action="store_true", help="large precision: integer-pipe products")
    ap.add_argument("--force-tensor", action="store_true", help="tensor-core products from 8 limbs up")
    ap.add_argument("--whole", action="store_true",
                    help="time whole transforms (CUDA events around execute_device) instead of per launch")
    a = ap.parse_args()
    if a.tier == "fp64":
        run_fp64(a)
        return
    if a.tier == "dd":
        run_dd(a)
        return
    if a.tier in ("qd", "ff"):
        run_multiword(a)
        return
    if a.tier == "queue":
        run_queue(a)
        return
    plan = M.MpPlan(a.n, a.prec, tensor="force" if a.force_tensor else not a.no_tensor)
    host = synthetic_planes(a.n, plan.limbs, plan.frac_bits, a.batch)
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    s = torch.cuda.current_stream().cuda_stream
    if a.whole:
        for _ in range(3):
            plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(a.reps, 20)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            plan.execute_device(a.batch, d_in.data_ptr(), d_out.data_ptr(), s)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        print(f"n={a.n} prec={a.prec} limbs={plan.limbs} batch={a.batch} whole transform {ms * 1e3:.1f} us "
              f"({a.batch / ms * 1e3:.0f} FFT/s)")
        return
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
