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
    launches_per_step = 1 + len(sched)

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
    level_bytes = [cnt * nn * 2 * L * 4 * 2 * B for (nn, cnt) in sched]  # read + write of touched points
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
        if len(cap["launches"]) == len(sched):
            traffic = sum(x["dram_read"] + x["dram_write"] for x in cap["launches"]) / len(sched) * B / cap["batch"]

    # ---- end to end through the C ABI with host mpfr_t arrays ----
    yr, yi = mparray.MpfrArray(n * B, p), mparray.MpfrArray(n * B, p)
    plan.execute(B, xr.ptr, xi.ptr, yr.ptr, yi.ptr)  # warm (pinned staging allocated here)
    e2e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plan.execute(B, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e = e2e_steps * B * world / dt

    # ---- accuracy of signal 0 against the 2P-bit oracle (CPU baseline leg) ----
    acc = {}
    if rank == 0 and world == 1 and not args.no_accuracy:
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
        acc = {"gpu_log2_rel_err": O.mp_errors(gr, gi, dr, di)["log2_rel"],
               "reference_log2_rel_err": O.mp_errors(rr, ri, dr, di)["log2_rel"],
               "bound_log2": O.mp_bound_log2(n, p), "oracle": f"direct DFT at {2 * p} bits, signal 0"}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    io_bytes = plan.words(B) * 4
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
        "roofline": {"bound": "hbm", "kernel": "mp_level_kernel", "achieved": ach_gbs, "peak": hbm_peak,
                     "unit": "GB/s", "frac": ach_gbs / hbm_peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": sum(level_bytes) / len(sched),
                     "traffic_source": "ncu dram__bytes_read+write, profiles/level_traffic_N1024_P1024_B2048.json",
                     "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)"},
        "roofline_compute": {"bound": "int32 multiply-add", "kernel": "mp_level_kernel",
                             "achieved": ach_prod / 1e12, "peak": prod_peak / 1e12,
                             "unit": "T limb-products/s", "frac": ach_prod / prod_peak,
                             "peak_source": f"measured live: IMAD {imad / 1e12:.2f} Tops/s, "
                                            f"IMAD.WIDE {imad_w / 1e12:.2f} Tops/s",
                             "work": "cmul(N) x ceil(P/32)^2 limb products"},
        "launch_ms": {"leaf": leaf_ms, "levels": dict(zip([s[0] for s in sched], level_ms))},
        "clocks": clk.summary(),
    }
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
