"""GPU parity tests of the FP64 path: bit-identical (0 ulp) to the reference's
double transform d_sr24_cp_fft (lab/serial/double/serial_d_fft6.c:93-429)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 64, 128, 1024, 4096, 1 << 16, 1 << 20])
def test_d_bitexact_vs_reference_restatement(M, orc, n):
    O = orc
    xr, xi = O.d_uniform(n, 100 + n)
    er, ei = O.DFFT(n)(xr, xi)
    yr, yi = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_fft(n, 1, 0, xr, xi, yr, yi) == M.OK, M.last_error()
    assert _bits_equal(yr, er) and _bits_equal(yi, ei)


@pytest.mark.parametrize("g", load_golden("d_"), ids=lambda g: g["name"])
def test_d_bitexact_vs_reference_golden(M, g):
    xr = np.array([float.fromhex(v) for v in g["inr"]])
    xi = np.array([float.fromhex(v) for v in g["ini"]])
    er = np.array([float.fromhex(v) for v in g["outr"]])
    ei = np.array([float.fromhex(v) for v in g["outi"]])
    n = g["N"]
    yr, yi = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_fft(n, 1, 0, xr, xi, yr, yi) == M.OK
    assert _bits_equal(yr, er) and _bits_equal(yi, ei)
    vr, vi = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_fft_v2(n, 0, 1, 0, xr, xi, vr, vi) == M.OK
    assert _bits_equal(vr, er) and _bits_equal(vi, ei)


def test_d_scaled_and_strided(M, orc):
    O = orc
    n, s = 2048, 2
    xr, xi = O.d_uniform(n * s, 3)
    yr, yi = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_fft(n, s, 0, xr, xi, yr, yi) == M.OK
    er, ei = O.DFFT(n)(np.ascontiguousarray(xr[::s]), np.ascontiguousarray(xi[::s]))
    assert _bits_equal(yr, er) and _bits_equal(yi, ei)
    sr, si = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_fft_scaled(n, s, 0, xr, xi, sr, si) == M.OK
    assert _bits_equal(sr, er / n) and _bits_equal(si, ei / n)


def test_d_batched_device_api(M, orc):
    import torch

    O = orc
    n, batch = 4096, 33
    xr = np.zeros((batch, n))
    xi = np.zeros((batch, n))
    for b in range(batch):
        xr[b], xi[b] = O.d_uniform(n, 500 + b)
    plan = M.DPlan(n)
    yr, yi = np.zeros_like(xr), np.zeros_like(xi)
    plan.execute(batch, xr, xi, yr, yi)
    f = O.DFFT(n)
    for b in range(batch):
        er, ei = f(xr[b], xi[b])
        assert _bits_equal(yr[b], er) and _bits_equal(yi[b], ei)
    # device layout [c][b][p]
    d_in = torch.from_numpy(np.stack([xr, xi]).copy()).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()
    assert _bits_equal(out[0], yr) and _bits_equal(out[1], yi)


@pytest.mark.parametrize("n", [1, 16, 1024, 65536])
def test_d_inverse_bitexact_vs_reference_procedure(M, orc, n):
    """d_sr24_cp_ifft is bit-identical to the reference's test() inverse:
    swap re/im, forward transform, swap back, divide by N
    (lab/serial/double/serial_d_fft6.c:511-524)."""
    O = orc
    xr, xi = O.d_uniform(n, 900 + n)
    fr, fi = O.DFFT(n)(xi, xr)           # forward of the swapped input
    er, ei = fi / n, fr / n              # swap back, divide by N
    yr, yi = np.zeros(n), np.zeros(n)
    assert M.d_sr24_cp_ifft(n, 1, 0, xr, xi, yr, yi) == M.OK
    assert _bits_equal(yr, er) and _bits_equal(yi, ei)
    plan = M.DPlan(n)
    zr, zi = np.zeros(n), np.zeros(n)
    plan.execute(1, xr, xi, zr, zi, scaled=True, inverse=True)
    assert _bits_equal(zr, er) and _bits_equal(zi, ei)
