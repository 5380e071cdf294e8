"""GPU parity at the precision-sweep and large-N configurations, through the C ABI.

* N=1024 at P = 512, 2048, 4096, 8192 bits with 129 signals per call: from
  2048 bits on the twiddle products run on the tensor cores in CTAs of 128
  signals, so 129 signals make two tiles, the second holding one signal.
  Every signal is checked against the reference's transform run at 2P bits
  (the oracle restates lab/serial/mp/serial_mp_fft3.c:121-253 bit for bit; its
  own error, about log2(N) 2^-2P, is negligible at P), and against the
  reference at P on the same inputs.  Signal 0 is also checked against the
  algorithm-independent direct DFT at 2P where that finishes in seconds.
* N = 2^14 and 2^16 directly against the reference at 2P (besides the
  swap-trick round trips of test_gpu_mp.py).
* The op counts of the GPU plan's own schedule: 7172 multiplications and
  27652 additions at N=1024 (lab/serial/mp/OPTIONS.md:42).

Acceptance as elsewhere: normwise relative error <= 8 log2(N) 2^-P and no
worse than the reference's own error at P plus half a bit.
"""
import concurrent.futures as cf
import os
import threading

import pytest

pytestmark = pytest.mark.gpu

MPFR_T = 32  # bytes per mpfr_t


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _slice(O, a, first, count, prec=None):
    out = O.MpArray(count, prec or a.prec)
    O.lib().orc_mp_copy(out.ptr, a.ptr + first * MPFR_T, count)
    return out


def _errors_vs_reference(O, n, p, xr, xi, yr, yi, signals):
    """(gpu, reference-at-P) log2 normwise errors of each signal against the
    reference at 2P, computed on the host cores (the oracle's C calls release
    the interpreter lock, each thread uses its own transform contexts)."""

    local = threading.local()

    def one(b):
        if not hasattr(local, "fft"):  # per-thread contexts: twiddle tables built once per thread
            local.fft = (O.MpFFT(n, 2 * p), O.MpFFT(n, p))
        sr, si = _slice(O, xr, b * n, n), _slice(O, xi, b * n, n)
        gr, gi = _slice(O, yr, b * n, n), _slice(O, yi, b * n, n)
        wr, wi = O.mp_pair(n, 2 * p)
        local.fft[0](sr, si, wr, wi)
        rr, ri = O.mp_pair(n, p)
        local.fft[1](sr, si, rr, ri)
        return b, O.mp_errors(gr, gi, wr, wi)["log2_rel"], O.mp_errors(rr, ri, wr, wi)["log2_rel"]

    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(one, signals))


@pytest.mark.parametrize("p", [512, 2048, 4096, 8192])
def test_mp_n1024_precision_sweep(M, orc, p):
    O = orc
    n, batch = 1024, 129
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 3000 + p)
    plan = M.MpPlan(n, p)
    yr, yi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    bound = O.mp_bound_log2(n, p)
    for b, e_gpu, e_ref in _errors_vs_reference(O, n, p, xr, xi, yr, yi, range(batch)):
        assert e_gpu <= bound, (p, b, e_gpu, bound)
        assert e_gpu <= e_ref + 0.5, (p, b, e_gpu, e_ref)
    if p <= 4096:  # the direct DFT at 2P bits for signal 0 (seconds at these sizes)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(_slice(O, xr, 0, n), _slice(O, xi, 0, n), dr, di)
        e = O.mp_errors(_slice(O, yr, 0, n), _slice(O, yi, 0, n), dr, di)["log2_rel"]
        assert e <= bound, (p, e, bound)


@pytest.mark.parametrize("n,p", [(1 << 14, 1024), (1 << 16, 256)])
def test_mp_large_n_vs_reference_at_2p(M, orc, n, p):
    O = orc
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 4000 + n)
    yr, yi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.OK, M.last_error()
    [(_, e_gpu, e_ref)] = _errors_vs_reference(O, n, p, xr, xi, yr, yi, [0])
    assert e_gpu <= O.mp_bound_log2(n, p), (e_gpu, O.mp_bound_log2(n, p))
    assert e_gpu <= e_ref + 0.5, (e_gpu, e_ref)


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 64, 256, 1024, 4096, 1 << 16])
def test_mp_plan_op_counts(M, orc, n):
    """Real multiplications and additions of the plan's own schedule equal the
    reference's counters on the same N (and the published 7172 / 27652 at
    N=1024)."""
    O = orc
    plan = M.MpPlan(n, 64)
    xr, xi = O.mp_pair(n, 64)
    O.fill_uniform(xr, xi, 1)
    yr, yi = O.mp_pair(n, 64)
    ref = O.MpFFT(n, 64)(xr, xi, yr, yi, count=True)[:2]
    assert plan.counts() == tuple(ref), (n, plan.counts(), ref)
    if n == 1024:
        assert plan.counts() == (7172, 27652)
