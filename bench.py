#!/usr/bin/env python
"""Benchmark: multiprecision FFTs per second at N=1024, P=1024 bits on B200.

One "step" = one batched transform of B signals (N=1024 points, P=1024-bit
re/im, uniform [-1,1) at full precision) through the chosen (batched) GPU
form.  Reported per the benchmark contract:

  value     whole-job FFT/s with the limb planes resident in HBM (device API),
            in+out buffers larger than L2 (no flush needed between steps)
  e2e       FFT/s through mpfft_mp_execute with HOST mpfr_t arrays: pack,
            H2D copy, kernels, D2H copy and unpack inside the timed region
  config    also carries the plain GPU path (one signal per call) and the
            normwise error of GPU and reference against a 2P-bit MPFR DFT
  roofline  HBM roofline of the dominant kernel (the L-butterfly level
            kernel); roofline_compute: the same kernel against the measured
            integer multiply-add peak, which is what bounds it
  cpu_baseline  the reference's own code (oracle/_ref, compiled from the
            reference sources), timed on this host's cores

--impl reference runs only the reference's CPU implementation (all host
cores, independent processes) and prints its line.

Multi-GPU (torchrun): every rank transforms its own batch (weak scaling, no
data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mp-FFT/s at N=1024,P=1024b: chosen vs plain GPU; max rel err vs 2P MPFR"
SEED = 20261203


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mpfft", choices=["mpfft", "reference"])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--prec", type=int, default=1024)
    ap.add_argument("--batch", type=int, default=2048, help="signals per GPU per step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra keys (other configurations, tiers, uneven batch, host roofline)")
    ap.add_argument("--dropin", action="store_true",
                    help="instead of the contract line: latency of one mp_sr24_cp_fft call (one signal of --n points "
                         "at --prec bits, host mpfr_t arrays) next to the reference's serial and OpenMP-4 code")
    ap.add_argument("--dropin-tier", default="mp", choices=["mp", "fp64"],
                    help="--dropin: mp_sr24_cp_fft (mp) or d_sr24_cp_fft on host double arrays (fp64)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# reference CPU implementation (oracle/_ref: the reference's own code files)
# ---------------------------------------------------------------------------

def _ref_worker(kind, n, p, m, seed):
    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    ref = O.Ref(kind, n, p)
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, seed)
    ref.mp_set_inputs(xr, xi)
    ref.run(1)
    ns, _ = ref.run(m)
    ref.free()
    return ns


def measure_reference(n: int, p: int, seconds: float, procs: int, steps: int = 1, warmup: int = 0):
    """Reference throughput on this host: `procs` independent processes each
    running the serial reference (lab/serial/mp/serial_mp_fft3.c), plus the
    OpenMP code mpFFT.c selects (lab/parallel/mp/parallel_mp_fft2.c, 4
    threads) run alone.  Returns FFT/s figures per step."""
    import multiprocessing as mp

    from oracle import oracle as O

    if not O.ref_available("mp_ser"):
        return None
    # calibrate m so one step of one worker takes about seconds/steps
    ns1 = _ref_worker("mp_ser", n, p, 3, SEED)
    t_one = ns1 / 3 / 1e9
    per_step = max(seconds / max(steps + warmup, 1), 0.5)
    m = max(1, int(per_step / t_one))
    ctx = mp.get_context("spawn")
    rates = []
    with ctx.Pool(procs) as pool:
        for s in range(warmup + steps):
            t0 = time.perf_counter()
            res = pool.starmap(_ref_worker, [("mp_ser", n, p, m, SEED + i) for i in range(procs)])
            wall = time.perf_counter() - t0
            if s >= warmup:
                rates.append(procs * m / (max(res) / 1e9))
    par = None
    if O.ref_available("mp_par"):
        mpar = max(1, int(min(per_step, 3.0) / t_one))
        ns = _ref_worker("mp_par", n, p, mpar, SEED)
        par = mpar / (ns / 1e9)
    return {"rates": rates, "m_per_proc": m, "procs": procs, "serial_fft_s": 1.0 / t_one, "omp4_fft_s": par}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    r = measure_reference(args.n, args.prec, seconds=max(20.0, 2.0 * (args.steps + args.warmup)), procs=procs,
                          steps=args.steps, warmup=args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent)"}))
        return
    value = statistics.median(r["rates"])
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "FFT/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "mpfr", "data": "synthetic",
        "config": {"workload": f"reference MPFR CP split-radix FFT N={args.n} P={args.prec} bits, "
                               f"{r['procs']} independent processes of lab/serial/mp/serial_mp_fft3.c"},
        "cpu_baseline": {"value": value, "unit": "FFT/s", "cores": r["procs"], "kind": "reference",
                         "sample": f"{r['procs']} processes x {r['m_per_proc']} transforms per step; "
                                   f"single core {r['serial_fft_s']:.1f} FFT/s; OpenMP-4 code "
                                   f"(parallel_mp_fft2.c) {r['omp4_fft_s']:.1f} FFT/s"},
        "e2e": {"value": value, "unit": "FFT/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic counts of the split-radix schedule
# ---------------------------------------------------------------------------

def level_mults(n: int) -> int:
    """Real multiplications in one node of size n (reference :203-236):
    k=0 none, k=n/8 four, every other k six."""
    q = n // 4
    if q <= 1:
        return 0
    return 4 + 6 * (q - 2)


def level_passes(sched, launch_ms):
    """The level launches of one transform: [(node sizes, points touched)].
    A level whose timed entry is 0 ran in one launch with the level below it
    (mp_level_pair_kernel: every node of size 2n with its first child, plus
    the nodes of size n that are not a first child, each point once)."""
    cnt = dict(sched)
    out = []
    for (nn, c), ms in zip(sched, launch_ms):
        if ms == 0.0 and out:
            lo = out[-1][0][0]
            out[-1] = ((lo, nn), cnt[nn] * nn + (cnt[lo] - cnt[nn]) * lo)
        else:
            out.append(((nn,), c * nn))
    return out


def dropin_arm(args):
    """One signal per call through the drop-in mp_sr24_cp_fft (the way the
    reference's own driver calls its transform, mpFFT.c:47): host mpfr_t arrays
    in and out, conversion, copies, kernels and synchronisation inside each
    call; wall time per call over many calls.  Beside it the reference's serial
    code (lab/serial/mp/serial_mp_fft3.c) and its OpenMP code
    (lab/parallel/mp/parallel_mp_fft2.c, 4 threads) on the same N and P."""
    import mpfft_b200 as M
    from mpfft_b200 import mparray
    from oracle import oracle as O

    if args.dropin_tier == "fp64":
        dropin_fp64(args)
        return
    n, p = args.n, args.prec
    xr, xi = mparray.MpfrArray(n, p), mparray.MpfrArray(n, p)
    mparray.fill_uniform(xr, xi, SEED)
    yr, yi = mparray.MpfrArray(n, p), mparray.MpfrArray(n, p)
    for _ in range(20):
        if M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) != M.OK:
            raise RuntimeError(M.last_error())
    reps = 300
    t0 = time.perf_counter()
    for _ in range(reps):
        M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    us = (time.perf_counter() - t0) / reps * 1e6
    ser = omp = None
    if O.ref_available("mp_ser"):
        t1 = _ref_worker("mp_ser", n, p, 3, SEED) / 3
        m = max(3, int(2e9 / t1))
        ser = _ref_worker("mp_ser", n, p, m, SEED) / m / 1e3
    if O.ref_available("mp_par"):
        m = max(3, int(1e9 / (ser * 1e3))) if ser else 3
        omp = _ref_worker("mp_par", n, p, m, SEED) / m / 1e3
    print(json.dumps({"metric": "drop-in call latency: one signal per mp_sr24_cp_fft call, host mpfr_t arrays",
                      "value": us, "unit": "us", "higher_is_better": False, "calls_per_s": 1e6 / us,
                      "config": {"n": n, "prec_bits": p, "calls": reps},
                      "reference_serial_us": ser, "reference_omp4_us": omp,
                      "speedup_vs_serial": (ser / us) if ser else None}))


def dropin_fp64(args):
    """One signal per d_sr24_cp_fft call (host double arrays, copies and
    synchronisation inside each call), the same transform on device-resident
    data (one signal per launch sequence, CUDA events), and the reference's
    serial double code (lab/serial/double/serial_d_fft6.c) on the host."""
    import numpy as np
    import torch

    import mpfft_b200 as M
    from oracle import oracle as O

    n = args.n
    rng = np.random.default_rng(SEED)
    xr, xi = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    yr, yi = np.zeros(n), np.zeros(n)
    for _ in range(10):
        if M.d_sr24_cp_fft(n, 1, 0, xr, xi, yr, yi) != M.OK:
            raise RuntimeError(M.last_error())
    reps = max(20, min(300, int(3e7 / n)))
    t0 = time.perf_counter()
    for _ in range(reps):
        M.d_sr24_cp_fft(n, 1, 0, xr, xi, yr, yi)
    us = (time.perf_counter() - t0) / reps * 1e6
    plan = M.DPlan(n)
    d_in = torch.from_numpy(np.concatenate([xr, xi])).cuda()
    d_out = torch.empty_like(d_in)
    st = torch.cuda.current_stream()
    for _ in range(10):
        plan.execute_device(1, d_in.data_ptr(), d_out.data_ptr(), stream=st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        plan.execute_device(1, d_in.data_ptr(), d_out.data_ptr(), stream=st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    dev_us = e0.elapsed_time(e1) / reps * 1e3
    ser = None
    if O.ref_available("d6"):
        ref = O.Ref("d6", n)
        ref.d_view(0)[:] = xr
        ref.d_view(1)[:] = xi
        t1 = ref.run(3)[0] / 3
        m = max(3, int(1e9 / max(t1, 1)))
        ser = ref.run(m)[0] / m / 1e3
        ref.free()
    print(json.dumps({"metric": "drop-in call latency: one signal per d_sr24_cp_fft call, host double arrays",
                      "value": us, "unit": "us", "higher_is_better": False, "config": {"n": n, "calls": reps},
                      "device_resident_us": dev_us, "reference_serial_us": ser,
                      "speedup_vs_serial": (ser / us) if ser else None}))


# ---------------------------------------------------------------------------
# accuracy of every signal of the step (after timing, on the host cores)
# ---------------------------------------------------------------------------

def worst_accuracy(n, p, B, xr, xi, yr, yi):
    """Normwise error of every one of the B GPU outputs against the
    reference's transform at 2P bits (lab/serial/mp/serial_mp_fft3.c restated
    by the oracle), and the reference's own error at P on the same inputs; on
    all host cores (the oracle's C calls release the interpreter lock)."""
    import concurrent.futures as cf

    from oracle import oracle as O

    L = O.lib()
    local = threading.local()

    def one(b):
        if not hasattr(local, "fft"):
            local.fft = (O.MpFFT(n, 2 * p), O.MpFFT(n, p))
        def cut(a):  # signal b of a batch of mpfr_t arrays
            t = O.MpArray(n, p)
            L.orc_mp_copy(t.ptr, a.ptr + b * n * 32, n)
            return t

        sr, si, gr, gi = cut(xr), cut(xi), cut(yr), cut(yi)
        wr, wi = O.mp_pair(n, 2 * p)
        local.fft[0](sr, si, wr, wi)
        rr, ri = O.mp_pair(n, p)
        local.fft[1](sr, si, rr, ri)
        return O.mp_errors(gr, gi, wr, wi)["log2_rel"], O.mp_errors(rr, ri, wr, wi)["log2_rel"]

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        res = list(ex.map(one, range(B)))
    worst = max(range(B), key=lambda b: res[b][0])
    bound = O.mp_bound_log2(n, p)
    return {"worst_gpu_log2_rel_err": res[worst][0], "worst_signal": worst,
            "reference_log2_rel_err_at_worst": res[worst][1],
            "worst_reference_log2_rel_err": max(r[1] for r in res),
            "signals_checked": B, "signals_over_bound": sum(r[0] > bound for r in res),
            "signals_worse_than_reference": sum(r[0] > r[1] + 0.5 for r in res),
            "accuracy_oracle": f"reference transform at {2 * p} bits, all {B} signals "
                               f"({time.perf_counter() - t0:.1f} s on {os.cpu_count()} host threads)"}


# ---------------------------------------------------------------------------
# extra keys: the other configurations, measured in the same run
# ---------------------------------------------------------------------------

def _cudart():
    """The CUDA runtime (plain copies into the uneven batch's device arenas)."""
    import ctypes as C
    import glob

    try:
        return C.CDLL("libcudart.so.12")
    except OSError:
        import torch

        d = os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib")
        return C.CDLL(sorted(glob.glob(os.path.join(d, "libcudart.so*")))[0])


def _time_device(fn, reps):
    """ms per call of fn() on the current stream, CUDA events, after 3 warm-up calls."""
    import torch

    for _ in range(3):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def host_bandwidth():
    """Host memory copy bandwidth over all cores (read + write bytes per
    second): the denominator of the end-to-end host roofline."""
    import concurrent.futures as cf

    import numpy as np

    nbytes = 1 << 30
    a = np.ones(nbytes // 8)
    b = np.empty_like(a)
    nt = os.cpu_count() or 1
    parts = np.array_split(np.arange(a.size), nt)
    sl = [slice(int(q[0]), int(q[-1]) + 1) for q in parts if q.size]

    def cp(s):
        np.copyto(b[s], a[s])

    with cf.ThreadPoolExecutor(max_workers=nt) as ex:
        list(ex.map(cp, sl))
        best = 1e30
        for _ in range(3):
            t0 = time.perf_counter()
            list(ex.map(cp, sl))
            best = min(best, time.perf_counter() - t0)
    return 2 * nbytes / best


def fill_uneven_arena(M, bp, ns, rng):
    """Synthetic inputs in a batch plan's input arena: uniform [-1,1) doubles
    (floats for float-float) in every floating signal, 5 % of them scaled by
    2^+-40, and random limbs with the top limb cleared (|A| < 2^F) in every
    limb signal.  Returns the number of points."""
    import ctypes as C

    import torch

    d_in, _, _ = bp.arenas()
    rt = _cudart()
    pat_d = torch.rand(1 << 21, dtype=torch.float64, device="cuda") * 2 - 1
    pat_f = pat_d.to(torch.float32)
    pat_i = torch.randint(-2**31, 2**31 - 1, (1 << 23,), dtype=torch.int32, device="cuda")
    sc = {40: pat_d * 2.0 ** 40, -40: pat_d * 2.0 ** -40}
    torch.cuda.synchronize()
    scales = rng.choice([0, 40, -40], len(ns), p=[0.9, 0.05, 0.05])
    points = 0
    for i, n in enumerate(ns):
        form, words, off, nb = bp.signal_format(i)
        points += n
        if form == M.FORM_LIMBS:
            src = pat_i
        elif form == M.FORM_FLOAT_FLOAT:
            src = pat_f
        else:
            src = sc.get(int(scales[i]), pat_d)
        rt.cudaMemcpy(C.c_void_p(d_in + off), C.c_void_p(src.data_ptr()), C.c_size_t(nb), 3)
        if form == M.FORM_LIMBS:  # the top limb planes of the real and imaginary parts
            top = (words - 1) * n * 4
            for c in (0, 1):
                rt.cudaMemset(C.c_void_p(d_in + off + c * words * n * 4 + top), 0, C.c_size_t(n * 4))
    rt.cudaDeviceSynchronize()
    return points


def measure_extras(args, e2e_fft_s, n, p):
    import numpy as np
    import torch

    import mpfft_b200 as M
    from mpfft_b200 import mparray
    from mpfft_b200.mparray import synthetic_planes

    out = {}
    st = torch.cuda.current_stream().cuda_stream

    def guard(key, fn):
        try:
            out[key] = fn()
        except Exception as e:  # recorded, not fatal: the contract line stands on its own
            out[key] = {"error": f"{type(e).__name__}: {e}"}

    # end-to-end host roofline: host memory traffic per transform / measured bandwidth
    def host_roofline():
        nl = (p + 63) // 64
        per_in = 32 + 8 * nl + (8 * nl + 9)            # mpfr_t struct, significand, staging write
        per_out = (8 * nl + 9) + 32 + 2 * 8 * nl + 32  # staging read, struct, significand RFO + write, struct write
        per_fft = 2 * n * (per_in + per_out)
        bw = host_bandwidth()
        return {"bytes_per_fft": per_fft, "bytes_per_component": per_in + per_out,
                "achieved_GBs": e2e_fft_s * per_fft / 1e9, "host_copy_GBs": bw / 1e9,
                "frac": e2e_fft_s * per_fft / bw,
                "note": "host memory bytes the mpfr_t gather/scatter must move per transform (in + out), "
                        "against a multi-threaded host copy; DMA traffic to pinned staging not counted"}

    guard("e2e_host_roofline", host_roofline)

    # configuration 1: one signal per drop-in call, N=1024, P=256, host mpfr_t arrays
    def dropin():
        nn, pp = 1024, 256
        xr, xi = mparray.MpfrArray(nn, pp), mparray.MpfrArray(nn, pp)
        mparray.fill_uniform(xr, xi, SEED)
        yr, yi = mparray.MpfrArray(nn, pp), mparray.MpfrArray(nn, pp)
        for _ in range(20):
            M.mp_sr24_cp_fft(nn, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        reps = 200
        t0 = time.perf_counter()
        for _ in range(reps):
            M.mp_sr24_cp_fft(nn, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        us = (time.perf_counter() - t0) / reps * 1e6
        r = {"workload": "mp_sr24_cp_fft, one signal per call, N=1024, P=256", "us_per_call": us}
        from oracle import oracle as O

        if O.ref_available("mp_ser"):
            ser = _ref_worker("mp_ser", nn, pp, 200, SEED) / 200 / 1e3
            r.update({"reference_serial_us": ser, "speedup": ser / us})
        return r

    guard("config1_dropin", dropin)

    # configuration 2: FP64 and double-double, 4096 signals x N=4096, and one FP64 signal of 2^20
    def fp64_dd():
        r = {}
        nn, bb = 4096, 4096
        g = torch.Generator(device="cuda").manual_seed(1)
        x = torch.rand((2, bb, nn), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        y = torch.empty_like(x)
        pl = M.DPlan(nn)
        ms = _time_device(lambda: pl.execute_device(bb, x.data_ptr(), y.data_ptr(), stream=st), 10)
        r["fp64_4096x4096"] = {"fft_per_s": bb / ms * 1e3, "ms": ms, "in_out_GBs": 2 * x.numel() * 8 / ms / 1e6}
        xd = torch.stack((x[0], x[0] * 2.0 ** -60, x[1], x[1] * 2.0 ** -60)).contiguous()
        yd = torch.empty_like(xd)
        dd = M.DDPlan(nn)
        ms = _time_device(lambda: dd.execute_device(bb, xd.data_ptr(), yd.data_ptr(), stream=st), 5)
        r["dd_4096x4096"] = {"fft_per_s": bb / ms * 1e3, "ms": ms, "in_out_GBs": 2 * xd.numel() * 8 / ms / 1e6}
        del x, y, xd, yd
        big = 1 << 20
        x1 = torch.rand((2, 1, big), dtype=torch.float64, device="cuda", generator=g)
        y1 = torch.empty_like(x1)
        p1 = M.DPlan(big)
        r["fp64_single_2^20_us"] = _time_device(lambda: p1.execute_device(1, x1.data_ptr(), y1.data_ptr(), stream=st),
                                                20) * 1e3
        return r

    guard("config2_fp64_dd", fp64_dd)

    # configuration 3: N=1024, batch 256, P = 64 .. 8192; tensor-core products from 35 limbs
    def sweep():
        r = {}
        tc = M.tc_int8_rate()
        imad = max(M.imad_rate(False) / 2, M.imad_rate(True))
        r["int8_tensor_macs_per_s"] = tc
        r["int_product_peak_per_s"] = imad
        for pp in (64, 128, 256, 512, 1024, 2048, 4096, 8192):
            nn, bb = 1024, 256
            pl = M.MpPlan(nn, pp)
            host = synthetic_planes(nn, pl.limbs, pl.frac_bits, bb, seed=pp)
            d_in = torch.from_numpy(host.view(np.int32)).cuda()
            d_out = torch.empty_like(d_in)
            ms = _time_device(lambda: pl.execute_device(bb, d_in.data_ptr(), d_out.data_ptr(), st), 3)
            fps = bb / ms * 1e3
            e = {"limbs": pl.limbs, "form": ["limbs", "tensor"][pl.form()], "fft_per_s": fps}
            if pl.form() == 1:  # byte products: cmul(N) (P/8)^2 per transform against the measured int8 rate
                e["tensor_frac"] = 7172 * (pp / 8) ** 2 * fps / tc
            else:
                e["int_frac"] = 7172 * ((pp + 31) // 32) ** 2 * fps / imad
            r[str(pp)] = e
            del d_in, d_out
        return r

    guard("config3_sweep", sweep)

    # the compensated tiers at N=4096 x 4096 signals (device resident)
    def tiers():
        r = {}
        nn, bb = 4096, 4096
        for t in ("ff", "qd"):
            pl = M.MultiwordPlan(nn, t)
            dt = torch.float32 if pl.word_bytes == 4 else torch.float64
            x = (torch.rand((2, pl.words, bb, nn), dtype=torch.float64, device="cuda") * 2 - 1).to(dt)
            x[:, 1:] *= 2.0 ** -60 if dt == torch.float64 else 2.0 ** -30
            y = torch.empty_like(x)
            ms = _time_device(lambda: pl.execute_device(bb, x.data_ptr(), y.data_ptr(), stream=st), 3)
            r[t] = {"fft_per_s": bb / ms * 1e3, "ms": ms}
            del x, y
        return r

    guard("tiers_4096x4096", tiers)

    # configuration 4: 10,000 signals, N log-uniform 2^4..2^16, P from {24, 53, 106, 212, 512, 1024}
    # (native tiers for the first four), 5 % scaled by 2^+-40 -- one graph launch
    def uneven():
        rng = np.random.default_rng(SEED)
        cnt = 10000
        ns = [1 << int(v) for v in rng.integers(4, 17, cnt)]
        ps = [int(v) for v in rng.choice([24, 53, 106, 212, 512, 1024], cnt)]
        t0 = time.perf_counter()
        bp = M.BatchPlan(ns, ps, float_tiers="native")
        t_plan = time.perf_counter() - t0
        points = fill_uneven_arena(M, bp, ns, rng)
        d_in, d_out, nbytes = bp.arenas()
        ms = _time_device(lambda: bp.execute_device(st), 5)
        r = {"signals": cnt, "points": points, "plan_s": t_plan, "ms": ms, "signals_per_s": cnt / ms * 1e3,
             "points_per_s": points / ms * 1e3, "arena_bytes": nbytes, "queues": bp.queues()}
        bp.autotune(save=False)
        ms2 = _time_device(lambda: bp.execute_device(st), 5)
        r.update({"autotuned_ms": ms2, "autotuned_queues": bp.queues()})
        bp.close()
        return r

    guard("config4_uneven", uneven)
    return out


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.dropin:
        if rank == 0:
            dropin_arm(args)
        return

    # CPU baseline before any CUDA work (spawned worker processes)
    base = None
    if rank == 0 and world == 1:
        base = measure_reference(args.n, args.prec, seconds=args.cpu_seconds, procs=os.cpu_count() or 1)

    import torch
    import torch.distributed as dist

    import mpfft_b200 as M
    from mpfft_b200 import mparray
    from mpfft_b200.dist import max_over_ranks, rank_seed

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    n, p, B = args.n, args.prec, args.batch
    plan = M.MpPlan(n, p)
    L = plan.limbs
    xr, xi = mparray.MpfrArray(n * B, p), mparray.MpfrArray(n * B, p)
    mparray.fill_uniform(xr, xi, rank_seed(SEED, rank))
    import numpy as np

    host = np.zeros(plan.words(B), dtype=np.uint32)
    exps = np.zeros(B, dtype=np.int64)
    plan.pack(B, xr.ptr, xi.ptr, host.ctypes.data, exps.ctypes.data)
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- chosen (batched) form, device resident ----
    # The clock sampler (200 ms period) starts with the warm-up, which runs
    # for at least W steps and at least ~1 s, so samples cover the load that
    # the timed steps run under.
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_w = time.perf_counter()
        done = 0
        while done < args.warmup or time.perf_counter() - t_w < 1.0:
            plan.execute_device(B, d_in.data_ptr(), d_out.data_ptr(), sh)
            done += 1
            if done % 8 == 0:
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute_device(B, d_in.data_ptr(), d_out.data_ptr(), sh)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms_max = max_over_ranks(e0.elapsed_time(e1), device="cuda")
    value = args.steps * B * world / (ms_max / 1e3)
    sched = plan.schedule()

    # ---- plain GPU path: one signal per call (device resident) ----
    n1 = plan.words(1)
    p_in, p_out = d_in[:n1].clone(), torch.empty(n1, dtype=torch.int32, device="cuda")
    # a real single-signal layout: signal 0 of the batch
    h1 = np.zeros(n1, dtype=np.uint32)
    e1x = np.zeros(1, dtype=np.int64)
    plan.pack(1, xr.ptr, xi.ptr, h1.ctypes.data, e1x.ctypes.data)
    p_in.copy_(torch.from_numpy(h1.view(np.int32)))
    for _ in range(3):
        plan.execute_device(1, p_in.data_ptr(), p_out.data_ptr(), sh)
    reps = 50
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        plan.execute_device(1, p_in.data_ptr(), p_out.data_ptr(), sh)
    e1.record(stream)
    torch.cuda.synchronize()
    plain = reps / (e0.elapsed_time(e1) / 1e3)

    # ---- per-launch attribution (roofline of the dominant kernel) ----
    per = [plan.execute_device_timed(B, d_in.data_ptr(), d_out.data_ptr(), sh) for _ in range(3)]
    avg = [statistics.mean(col) for col in zip(*per)]
    leaf_ms, level_ms = avg[0], avg[1:]
    passes = level_passes(sched, per[0][1:])
    launches_per_step = 1 + len(passes)
    # read + write of the points each launch touches
    level_bytes = [pts * 2 * L * 4 * 2 * B for (_, pts) in passes]
    level_prods = [cnt * level_mults(nn) * B * ((p + 31) // 32) ** 2 for (nn, cnt) in sched]
    lvl_time = sum(level_ms) / 1e3
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    ach_gbs = sum(level_bytes) / lvl_time / 1e9
    imad = M.imad_rate(False)
    imad_w = M.imad_rate(True)
    prod_peak = max(imad / 2, imad_w)  # one 32x32->64 product = lo+hi multiply-adds, or one wide
    ach_prod = sum(level_prods) / lvl_time
    # DRAM traffic of the level launches from the committed ncu capture of this
    # workload (one-pass metrics), per launch like `achieved`, scaled by batch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"level_traffic_N{n}_P{p}_B2048.json")
    if os.path.exists(tpath):
        cap = json.load(open(tpath))
        if len(cap["launches"]) == len(passes):
            traffic = sum(x["dram_read"] + x["dram_write"] for x in cap["launches"]) / len(passes) * B / cap["batch"]

    # ---- end to end through the C ABI with host mpfr_t arrays ----
    yr, yi = mparray.MpfrArray(n * B, p), mparray.MpfrArray(n * B, p)
    plan.execute(B, xr.ptr, xi.ptr, yr.ptr, yi.ptr)  # warm (pinned staging allocated here)
    e2e_steps = args.steps
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plan.execute(B, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e = e2e_steps * B * world / dt

    # ---- accuracy against the oracle (CPU baseline leg, after timing) ----
    acc = {}
    if rank == 0 and world == 1 and not args.no_accuracy:
        acc.update(worst_accuracy(n, p, B, xr, xi, yr, yi))
        from oracle import oracle as O

        gr, gi = O.mp_pair(n, p)
        sr, si = O.mp_pair(n, p)
        O.lib().orc_mp_copy(sr.ptr, xr.ptr, n)
        O.lib().orc_mp_copy(si.ptr, xi.ptr, n)
        O.lib().orc_mp_copy(gr.ptr, yr.ptr, n)
        O.lib().orc_mp_copy(gi.ptr, yi.ptr, n)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(sr, si, dr, di)
        rr, ri = O.mp_pair(n, p)
        O.MpFFT(n, p)(sr, si, rr, ri)
        acc.update({"gpu_log2_rel_err": O.mp_errors(gr, gi, dr, di)["log2_rel"],
               "reference_log2_rel_err": O.mp_errors(rr, ri, dr, di)["log2_rel"],
               "bound_log2": O.mp_bound_log2(n, p), "oracle": f"direct DFT at {2 * p} bits, signal 0"})

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras = measure_extras(args, e2e, n, p)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    io_bytes = plan.words(B) * 4
    level_kernel = ("mp_level_pair_kernel (two levels per launch)"
                    if any(len(lv) == 2 for lv, _ in passes) else "mp_level_kernel")
    line = {
        "metric": METRIC, "value": value, "unit": "FFT/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: re/im iid uniform[-1,1) at full P, seeded MT19937",
        "config": {
            "workload": f"mp conjugate-pair split-radix FFT, N={n}, P={p} bits, batch {B} per GPU",
            "n": n, "prec_bits": p, "batch_per_gpu": B, "limbs": L, "frac_bits": plan.frac_bits,
            "l2": f"in+out buffers {2 * io_bytes / 2**20:.0f} MiB > 126 MB L2, no flush",
            "plain_gpu_fft_per_s": plain, "chosen_vs_plain": value / world / plain, **acc,
        },
        "e2e": {"value": e2e, "unit": "FFT/s", "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": level_kernel, "achieved": ach_gbs, "peak": hbm_peak,
                     "unit": "GB/s", "frac": ach_gbs / hbm_peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": sum(level_bytes) / len(passes),
                     "traffic_source": "ncu dram__bytes_read+write, profiles/level_traffic_N1024_P1024_B2048.json",
                     "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)"},
        "roofline_compute": {"bound": "int32 multiply-add", "kernel": level_kernel,
                             "achieved": ach_prod / 1e12, "peak": prod_peak / 1e12,
                             "unit": "T limb-products/s", "frac": ach_prod / prod_peak,
                             "peak_source": f"measured live: IMAD {imad / 1e12:.2f} Tops/s, "
                                            f"IMAD.WIDE {imad_w / 1e12:.2f} Tops/s",
                             "work": "cmul(N) x ceil(P/32)^2 limb products"},
        "launch_ms": {"leaf": leaf_ms, "levels": dict(zip([s[0] for s in sched], level_ms))},
        "clocks": clk.summary(),
    }
    if extras:
        line["extras"] = extras
    if base:
        line["cpu_baseline"] = {
            "value": statistics.median(base["rates"]), "unit": "FFT/s", "cores": base["procs"], "kind": "reference",
            "sample": f"{base['procs']} processes x {base['m_per_proc']} transforms of serial_mp_fft3.c; "
                      f"single core {base['serial_fft_s']:.1f} FFT/s; OpenMP-4 parallel_mp_fft2.c "
                      f"{base['omp4_fft_s']:.1f} FFT/s"}
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
