"""GPU parity tests of the multiprecision path, through the C ABI.

Acceptance: normwise relative error max_k max(|dRe|,|dIm|) / max_k |X_k|_inf
against a direct MPFR DFT at 2P bits must be <= 8*log2(N)*2^-P, and no worse
than the reference's own transform at the same P on the same inputs.
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _inputs(O, n, p, seed, scale=0):
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, seed)
    if scale:
        O.lib().orc_mp_scale2(xr.ptr, n, scale)
        O.lib().orc_mp_scale2(xi.ptr, n, scale)
    return xr, xi


def _gpu(M, O, xr, xi, n, p, fn="mp_sr24_cp_fft"):
    yr, yi = O.mp_pair(n, p)
    code = getattr(M, fn)(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    assert code == M.OK, M.last_error()
    return yr, yi


@pytest.mark.parametrize(
    "n,p",
    [(1, 64), (2, 64), (4, 64), (8, 64), (16, 64), (32, 128), (64, 256), (128, 53), (256, 1024), (512, 512),
     (1024, 64), (1024, 256), (2048, 128)],
)
def test_mp_matches_2p_dft_oracle(M, orc, n, p):
    O = orc
    xr, xi = _inputs(O, n, p, 1000 + n)
    yr, yi = _gpu(M, O, xr, xi, n, p)
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft(xr, xi, dr, di)
    e_gpu = O.mp_errors(yr, yi, dr, di)
    bound = O.mp_bound_log2(n, p)
    assert e_gpu["log2_rel"] <= bound, (e_gpu, bound)
    # the reference's own transform on the same inputs, same P
    rr, ri = O.mp_pair(n, p)
    O.MpFFT(n, p)(xr, xi, rr, ri)
    e_ref = O.mp_errors(rr, ri, dr, di)
    assert e_gpu["log2_rel"] <= e_ref["log2_rel"] + 0.5, (e_gpu, e_ref)


@pytest.mark.parametrize("g", load_golden("mp_"), ids=lambda g: g["name"])
def test_mp_matches_reference_golden(M, orc, g):
    O = orc
    n, p = g["N"], g["P"]
    xr, xi = O.mp_pair(n, p)
    xr.set_hex(g["inr"])
    xi.set_hex(g["ini"])
    rr, ri = O.mp_pair(n, p)
    rr.set_hex(g["outr"])
    ri.set_hex(g["outi"])
    yr, yi = _gpu(M, O, xr, xi, n, p)
    e = O.mp_errors(yr, yi, rr, ri)
    assert e["log2_rel"] <= O.mp_bound_log2(n, p), e


def test_mp_v2_and_scaled(M, orc):
    O = orc
    n, p = 256, 192
    xr, xi = _inputs(O, n, p, 7)
    yr, yi = _gpu(M, O, xr, xi, n, p)
    vr, vi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft_v2(n, 0, 1, 0, xr.ptr, xi.ptr, vr.ptr, vi.ptr) == M.OK
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, vr.ptr, n) == 0 and L.orc_mp_count_diff(yi.ptr, vi.ptr, n) == 0
    sr, si = _gpu(M, O, xr, xi, n, p, fn="mp_sr24_cp_fft_scaled")
    L.orc_mp_scale2(yr.ptr, n, -8)
    L.orc_mp_scale2(yi.ptr, n, -8)
    assert L.orc_mp_count_diff(yr.ptr, sr.ptr, n) == 0 and L.orc_mp_count_diff(yi.ptr, si.ptr, n) == 0


@pytest.mark.parametrize("n,p,batch", [(128, 256, 5), (128, 1024, 32), (64, 100, 64), (16, 64, 256), (64, 512, 128),
                                       (32, 960, 128)])
def test_mp_batch_equals_single_calls(M, orc, n, p, batch):
    """Batched and single-signal calls are bit-equal.  In a batch that is a
    multiple of 32 every warp shares one butterfly index; in a multiple of 128
    (3, 17 and 31 limbs here) every CTA does, and the level kernel stages its
    twiddles in shared memory; single signals read them from global memory."""
    O = orc
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 31)
    L = O.lib()
    # make the signals differ in scale
    for b in range(batch):
        e = (0, 40, -40, 3, 0)[b % 5]
        for a in (xr, xi):
            L.orc_mp_scale2(a.ptr + b * n * 32, n, e)
    plan = M.MpPlan(n, p)
    yr, yi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    for b in range(batch):
        sr, si = O.mp_pair(n, p)
        assert M.mp_sr24_cp_fft(n, 1, 0, xr.ptr + b * n * 32, xi.ptr + b * n * 32, sr.ptr, si.ptr) == M.OK
        assert L.orc_mp_count_diff(sr.ptr, yr.ptr + b * n * 32, n) == 0
        assert L.orc_mp_count_diff(si.ptr, yi.ptr + b * n * 32, n) == 0


# 34, 33, 32, 31, 30, 17, 4 and 2 limbs at N=1024: both sides of the
# two-registers-per-lane boundary of the warp kernel's columns (L+2 > 32) and
# of its limbs (L > 32)
@pytest.mark.parametrize("p", [1060, 1024, 980, 950, 920, 512, 100, 24])
def test_mp_small_batch_level_kernel_bit_identical(M, p):
    """Level launches with few butterflies run each product across a warp
    (mp_level_warp_kernel, single signals at N=1024: at most 256 butterflies
    per level); launches below one wave of the main level kernel run one
    thread per product (mp_level_small_kernel).  On the same limb planes, a
    batch of 2048 signals at N=1024 (every level pair in one launch of
    mp_level_pair_kernel) and
    single signals cut from it give bit-identical outputs, and so do batches
    of 16 (levels of up to 4096 butterflies)."""
    import torch

    from mpfft_b200.mparray import synthetic_planes

    n, B = 1024, 2048
    plan = M.MpPlan(n, p)
    Lm = plan.limbs
    host = synthetic_planes(n, Lm, plan.frac_bits, B, seed=3)
    s = torch.cuda.current_stream().cuda_stream
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute_device(B, d_in.data_ptr(), d_out.data_ptr(), s)
    torch.cuda.synchronize()
    big = d_out.cpu().numpy().view(np.uint32).reshape(2, Lm, n, B)
    planes = host.reshape(2, Lm, n, B)
    for b in (0, 1, 1000, B - 1):
        one = np.ascontiguousarray(planes[:, :, :, b]).reshape(-1)
        d1 = torch.from_numpy(one.view(np.int32)).cuda()
        o1 = torch.empty_like(d1)
        plan.execute_device(1, d1.data_ptr(), o1.data_ptr(), s)
        torch.cuda.synchronize()
        assert np.array_equal(o1.cpu().numpy().view(np.uint32).reshape(2, Lm, n), big[:, :, :, b]), b
    sub = np.ascontiguousarray(planes[:, :, :, 100:116]).reshape(-1)
    d16 = torch.from_numpy(sub.view(np.int32)).cuda()
    o16 = torch.empty_like(d16)
    plan.execute_device(16, d16.data_ptr(), o16.data_ptr(), s)
    torch.cuda.synchronize()
    assert np.array_equal(o16.cpu().numpy().view(np.uint32).reshape(2, Lm, n, 16), big[:, :, :, 100:116])


# (n, precision, batch): 33 limbs (rolled combine loop) and 9, 10, 17, 25
# limbs (unrolled); batches that are not a multiple of the CTA size, so one
# CTA holds fused and unfused butterflies; n = 2048 has an odd number of
# levels (the top one runs alone); n = 16 is one level pair and nothing else.
# Each batch gives every pair at least one wave of fused threads.
@pytest.mark.parametrize("n,p,B", [(1024, 1024, 1000), (1024, 512, 1200), (1024, 760, 2000), (2048, 256, 900),
                                   (16, 1024, 40000), (64, 300, 20000)])
def test_mp_level_pairs_bit_identical(M, n, p, B):
    """Batches large enough for the main level kernel run two levels per
    launch (mp_level_pair_kernel: each node with its first child, the child's
    outputs fed into the parent's combine without a store).  Single signals
    cut from the batch run every level on its own (warp-parallel and
    small-batch kernels): the outputs are bit-identical."""
    import torch

    from mpfft_b200.mparray import synthetic_planes

    plan = M.MpPlan(n, p)
    Lm = plan.limbs
    host = synthetic_planes(n, Lm, plan.frac_bits, B, seed=11)
    s = torch.cuda.current_stream().cuda_stream
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    ms = plan.execute_device_timed(B, d_in.data_ptr(), d_out.data_ptr(), s)
    torch.cuda.synchronize()
    assert ms[1:].count(0.0) == len(ms[1:]) // 2, "not every level pair ran as one launch"
    big = d_out.cpu().numpy().view(np.uint32).reshape(2, Lm, n, B)
    planes = host.reshape(2, Lm, n, B)
    for b in (0, 127, 128, B // 2, B - 1):
        one = np.ascontiguousarray(planes[:, :, :, b]).reshape(-1)
        d1 = torch.from_numpy(one.view(np.int32)).cuda()
        o1 = torch.empty_like(d1)
        plan.execute_device(1, d1.data_ptr(), o1.data_ptr(), s)
        torch.cuda.synchronize()
        assert np.array_equal(o1.cpu().numpy().view(np.uint32).reshape(2, Lm, n), big[:, :, :, b]), b


def test_mp_device_api_matches_host_api(M, orc):
    import torch

    O = orc
    n, p, batch = 256, 128, 64
    plan = M.MpPlan(n, p)
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 5)
    host = np.zeros(plan.words(batch), dtype=np.uint32)
    exps = np.zeros(batch, dtype=np.int64)
    plan.pack(batch, xr.ptr, xi.ptr, host.ctypes.data, exps.ctypes.data)
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(np.uint32).copy()
    yr, yi = O.mp_pair(n * batch, p)
    plan.unpack(batch, out.ctypes.data, exps.ctypes.data, yr.ptr, yi.ptr)
    zr, zi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0


def test_mp_edge_inputs(M, orc):
    O = orc
    L = O.lib()
    n, p = 64, 128
    # all zero -> all zero
    xr, xi = O.mp_pair(n, p)
    yr, yi = _gpu(M, O, xr, xi, n, p)
    assert np.all(yr.to_double() == 0) and np.all(yi.to_double() == 0)
    # unit impulse at 0 -> all ones, exactly
    L.orc_mp_set_ui(xr.ptr, 1, 1)
    yr, yi = _gpu(M, O, xr, xi, n, p)
    ones, zeros = O.mp_pair(n, p)
    L.orc_mp_set_ui(ones.ptr, n, 1)
    assert L.orc_mp_count_diff(yr.ptr, ones.ptr, n) == 0
    assert L.orc_mp_count_diff(yi.ptr, zeros.ptr, n) == 0
    # extreme block exponents: error relative to the signal's own scale
    for sc in (40, -40, 1000, -1000):
        xr, xi = _inputs(O, n, p, 3, scale=sc)
        yr, yi = _gpu(M, O, xr, xi, n, p)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(xr, xi, dr, di)
        assert O.mp_errors(yr, yi, dr, di)["log2_rel"] <= O.mp_bound_log2(n, p)


def test_mp_strided_input(M, orc):
    O = orc
    n, p, s = 128, 96, 3
    xr, xi = O.mp_pair(n * s, p)
    O.fill_uniform(xr, xi, 9)
    yr, yi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft(n, s, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.OK
    gr, gi = O.mp_pair(n, p)
    O.lib().orc_mp_gather(gr.ptr, xr.ptr, n, s)
    O.lib().orc_mp_gather(gi.ptr, xi.ptr, n, s)
    zr, zi = _gpu(M, O, gr, gi, n, p)
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n) == 0 and L.orc_mp_count_diff(yi.ptr, zi.ptr, n) == 0


def test_mp_nonfinite_input_reports_error(M, orc):
    O = orc
    n, p = 32, 64
    xr, xi = _inputs(O, n, p, 1)
    O.lib().orc_mp_set_inf(xr.ptr, 3, 1)
    yr, yi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.ENONFINITE
    assert np.all(np.isnan(yr.to_double()))


@pytest.mark.parametrize("n,p", [(1 << 16, 256), (1 << 14, 1024)])
def test_mp_large_n_roundtrip(M, orc, n, p):
    """Size-independent property at full sizes: the inverse by the swap trick
    (the reference's test(), parallel_mp_fft2.c:441-473) returns the input
    within the error bound of two transforms."""
    O = orc
    xr, xi = _inputs(O, n, p, 17)
    yr, yi = _gpu(M, O, xr, xi, n, p)
    zr, zi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft_scaled(n, 1, 0, yi.ptr, yr.ptr, zr.ptr, zi.ptr) == M.OK
    e = O.mp_errors(zi, zr, xr, xi)
    assert e["log2_rel"] <= O.mp_bound_log2(n, p) + 1, e


@pytest.mark.parametrize("n,p_in,p_out,batch,scaled", [
    (1024, 1024, 1024, 64, False), (256, 100, 64, 33, False), (64, 53, 200, 32, True), (16, 64, 64, 3, False),
    (2, 64, 30, 5, True)])
def test_mp_gpu_conversion_matches_host_conversion(M, orc, n, p_in, p_out, batch, scaled):
    """The GPU import/export of significands gives bit-identical outputs to the
    host conversion (mpfr_set_z_2exp rounding), incl. rounding to a lower output
    precision, zero signals, negative values and 2^+-40 block scales."""
    O = orc
    L = O.lib()
    prec = max(p_in, p_out)
    xr, xi = O.mp_pair(n * batch, p_in)
    O.fill_uniform(xr, xi, 77)
    for b in range(batch):
        e = (0, 40, -40, 7, 0)[b % 5]
        for a in (xr, xi):
            L.orc_mp_scale2(a.ptr + b * n * 32, n, e)
    if batch > 1:  # signal 1 entirely zero
        L.orc_mp_set_ui(xr.ptr + n * 32, n, 0)
        L.orc_mp_set_ui(xi.ptr + n * 32, n, 0)
    gpu = M.MpPlan(n, prec)
    host = M.MpPlan(n, prec, host_conversion=True)
    yr, yi = O.mp_pair(n * batch, p_out)
    zr, zi = O.mp_pair(n * batch, p_out)
    gpu.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr, scaled=scaled)
    host.execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr, scaled=scaled)
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0


@pytest.mark.parametrize("what,sig", [("input", 5), ("input", 300), ("output", 520), ("output", 0)])
def test_mp_precision_change_mid_batch(M, orc, what, sig):
    """A batch whose precisions change part way (input limb count or output
    precision of one signal): the GPU-conversion pipeline (chunks of 256
    signals here) completes the chunks before the change and the remaining
    signals are converted on the host; every output is bit-identical to a
    host-conversion plan's."""
    O = orc
    L = O.lib()
    n, p, batch = 16, 128, 600
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 91)
    yr, yi = O.mp_pair(n * batch, p)
    zr, zi = O.mp_pair(n * batch, p)
    off = sig * n * 32
    if what == "input":
        for a in (xr, xi):
            L.orc_mp_set_prec_all(a.ptr + off, n, 300)
        L.orc_mp_fill_uniform(xr.ptr + off, xi.ptr + off, n, 7)
    else:
        for a in (yr, yi, zr, zi):
            L.orc_mp_set_prec_all(a.ptr + off, n, 100)
    gpu = M.MpPlan(n, p)
    host = M.MpPlan(n, p, host_conversion=True)
    gpu.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    host.execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0


@pytest.mark.parametrize("n,p", [(256, 256), (1024, 1024), (4, 64)])
def test_mp_inverse_entry(M, orc, n, p):
    """mp_sr24_cp_ifft = the reference's test() inverse (swap, forward, swap,
    divide by N); against the 2P-bit inverse DFT and as a round trip."""
    O = orc
    L = O.lib()
    xr, xi = _inputs(O, n, p, 41)
    yr, yi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_ifft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.OK
    # 2P oracle of the inverse: (1/n) swap(DFT(swap(x)))
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft(xi, xr, di, dr)
    L.orc_mp_scale2(dr.ptr, n, -int(math.log2(n)))
    L.orc_mp_scale2(di.ptr, n, -int(math.log2(n)))
    assert O.mp_errors(yr, yi, dr, di)["log2_rel"] <= O.mp_bound_log2(n, p)
    # forward of the inverse returns the input
    zr, zi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft(n, 1, 0, yr.ptr, yi.ptr, zr.ptr, zi.ptr) == M.OK
    assert O.mp_errors(zr, zi, xr, xi)["log2_rel"] <= O.mp_bound_log2(n, p) + 1
    # batched flag gives the same result
    plan = M.MpPlan(n, p)
    wr, wi = O.mp_pair(n, p)
    plan.execute(1, xr.ptr, xi.ptr, wr.ptr, wi.ptr, scaled=True, inverse=True)
    assert L.orc_mp_count_diff(wr.ptr, yr.ptr, n) == 0 and L.orc_mp_count_diff(wi.ptr, yi.ptr, n) == 0


@pytest.mark.parametrize("n,p,batch", [(16, 2048, 1), (64, 2048, 32), (16, 4096, 2), (8, 8192, 1), (256, 1100, 1),
                                     (1, 1100, 3), (2, 2048, 1), (4, 9000, 2)])
def test_mp_large_precision(M, orc, n, p, batch):
    """Precisions beyond the register kernels (L > 34 limbs) run the streaming
    kernels: same error bound against the 2P-bit DFT, no worse than the
    reference at the same P; host-array, batched and conversion paths agree."""
    O = orc
    L = O.lib()
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 55 + p)
    plan = M.MpPlan(n, p)
    assert plan.limbs > 34
    yr, yi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    zr, zi = O.mp_pair(n * batch, p)
    M.MpPlan(n, p, host_conversion=True).execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0 and L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0
    for b in (0, batch - 1):
        sr, si = O.mp_pair(n, p)
        L.orc_mp_copy(sr.ptr, xr.ptr + b * n * 32, n)
        L.orc_mp_copy(si.ptr, xi.ptr + b * n * 32, n)
        gr, gi = O.mp_pair(n, p)
        L.orc_mp_copy(gr.ptr, yr.ptr + b * n * 32, n)
        L.orc_mp_copy(gi.ptr, yi.ptr + b * n * 32, n)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(sr, si, dr, di)
        e_gpu = O.mp_errors(gr, gi, dr, di)["log2_rel"]
        rr, ri = O.mp_pair(n, p)
        O.MpFFT(n, p)(sr, si, rr, ri)
        e_ref = O.mp_errors(rr, ri, dr, di)["log2_rel"]
        assert e_gpu <= O.mp_bound_log2(n, p) and e_gpu <= e_ref + 0.5, (e_gpu, e_ref)
