"""GPU tests of the multi-dimensional transforms (iterated one-dimensional
transforms over row-major signals).

mp: against a 2P-bit direct DFT along every axis, bound 8*log2(N)*2^-P with N
the total point count; batches, conversion paths and the device entry agree
bit for bit.  FP64: bit-identical to applying the reference's double
transform (our restatement, itself pinned bit-exact to the reference) along
the last axis, then the next, ..., then the first.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MPFR_T = 32


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _prod(dims):
    return int(np.prod(dims))


@pytest.mark.parametrize("dims,p", [((4, 8), 128), ((16, 32), 256), ((2, 4, 8), 192), ((32, 64), 64),
                                    ((1, 16), 100), ((16, 1), 100), ((8, 8), 2048), ((4, 4, 4), 1024)])
def test_mp_nd_matches_2p_oracle(M, orc, dims, p):
    O = orc
    n = _prod(dims)
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 17 + n)
    plan = M.MpPlanND(dims, p)
    yr, yi = O.mp_pair(n, p)
    plan.execute(1, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft_nd(dims, xr, xi, dr, di)
    e = O.mp_errors(yr, yi, dr, di)["log2_rel"]
    assert e <= O.mp_bound_log2(n, p), e


@pytest.mark.parametrize("dims,p,batch", [((8, 16), 256, 5), ((4, 2, 8), 64, 33), ((2, 32), 1100, 3)])
def test_mp_nd_batch_paths_agree(M, orc, dims, p, batch):
    """Batched = single calls; GPU conversion = host conversion; device limb
    planes (pack -> execute_device -> unpack) = host arrays; bit for bit."""
    import torch

    O = orc
    L = O.lib()
    n = _prod(dims)
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 3)
    if batch > 2:
        L.orc_mp_scale2(xr.ptr + 2 * n * MPFR_T, n, 40)
        L.orc_mp_scale2(xi.ptr + 2 * n * MPFR_T, n, 40)
    plan = M.MpPlanND(dims, p)
    yr, yi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    zr, zi = O.mp_pair(n * batch, p)
    M.MpPlanND(dims, p, host_conversion=True).execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0
    for b in (0, batch - 1):
        sr, si = O.mp_pair(n, p)
        plan.execute(1, xr.ptr + b * n * MPFR_T, xi.ptr + b * n * MPFR_T, sr.ptr, si.ptr)
        assert L.orc_mp_count_diff(sr.ptr, yr.ptr + b * n * MPFR_T, n) == 0
        assert L.orc_mp_count_diff(si.ptr, yi.ptr + b * n * MPFR_T, n) == 0
    planes = np.zeros(plan.words(batch), dtype=np.uint32)
    exps = np.zeros(batch, dtype=np.int64)
    plan.pack(batch, xr.ptr, xi.ptr, planes.ctypes.data, exps.ctypes.data)
    d_in = torch.from_numpy(planes.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(np.uint32).copy()
    wr, wi = O.mp_pair(n * batch, p)
    plan.unpack(batch, out.ctypes.data, exps.ctypes.data, wr.ptr, wi.ptr)
    assert L.orc_mp_count_diff(wr.ptr, yr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(wi.ptr, yi.ptr, n * batch) == 0


def test_mp_nd_inverse_roundtrip(M, orc):
    O = orc
    dims, p = (16, 8, 4), 320
    n = _prod(dims)
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 9)
    plan = M.MpPlanND(dims, p)
    yr, yi = O.mp_pair(n, p)
    plan.execute(1, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    zr, zi = O.mp_pair(n, p)
    plan.execute(1, yr.ptr, yi.ptr, zr.ptr, zi.ptr, scaled=True, inverse=True)
    assert O.mp_errors(zr, zi, xr, xi)["log2_rel"] <= O.mp_bound_log2(n, p) + 1


def _d_axis(O, xr, xi, axis):
    """The oracle double transform along one axis of an nd array."""
    xr, xi = np.moveaxis(xr, axis, -1), np.moveaxis(xi, axis, -1)
    shp = xr.shape
    fr, fi = xr.reshape(-1, shp[-1]).copy(), xi.reshape(-1, shp[-1]).copy()
    f = O.DFFT(shp[-1])
    for r in range(fr.shape[0]):
        fr[r], fi[r] = f(np.ascontiguousarray(fr[r]), np.ascontiguousarray(fi[r]))
    return np.moveaxis(fr.reshape(shp), -1, axis), np.moveaxis(fi.reshape(shp), -1, axis)


@pytest.mark.parametrize("dims,batch", [((64, 128), 3), ((8, 16, 32), 2), ((4096, 2), 1), ((1, 256), 2),
                                        ((256, 256), 1)])
def test_d_nd_bitexact_vs_axis_by_axis_reference(M, orc, dims, batch):
    O = orc
    rng = np.random.default_rng(5)
    xr = rng.uniform(-1, 1, size=(batch,) + dims)
    xi = rng.uniform(-1, 1, size=(batch,) + dims)
    er, ei = xr.copy(), xi.copy()
    for b in range(batch):
        a, c = er[b], ei[b]
        for axis in reversed(range(len(dims))):
            a, c = _d_axis(O, a, c, axis)
        er[b], ei[b] = a, c
    plan = M.DPlanND(dims)
    yr, yi = np.zeros_like(xr), np.zeros_like(xi)
    plan.execute(batch, xr, xi, yr, yi)
    assert np.array_equal(yr.view(np.uint64), er.view(np.uint64))
    assert np.array_equal(yi.view(np.uint64), ei.view(np.uint64))
    sr, si = np.zeros_like(xr), np.zeros_like(xi)
    plan.execute(batch, xr, xi, sr, si, scaled=True)
    n = _prod(dims)
    assert np.array_equal(sr.view(np.uint64), (er / n).view(np.uint64))
    # and within rounding of numpy's transform
    ref = np.fft.fftn(xr + 1j * xi, axes=tuple(range(1, len(dims) + 1)))
    assert np.max(np.abs(yr + 1j * yi - ref)) <= 1e-12 * np.max(np.abs(ref))
