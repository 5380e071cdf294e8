"""GPU tests of the compensated floating-point tiers and of the dispatch of
mp plans to them.

* quad-double (about 212 bits) against a 424-bit oracle: the direct DFT up to
  N = 4096, the reference's transform at 424 bits above;
* float-float (about 48 bits) against a 96-bit direct DFT;
* device entry = host entry bit for bit; scaled = unscaled / N exactly;
  inverse of the forward returns the input;
* MPFFT_PLAN_FLOAT_TIERS: each precision lands on the documented tier, meets
  the multiprecision contract 8 log2(N) 2^-P against the 2P-bit oracle, and
  inputs outside a tier's exponent window run on the limbs (bit-identical to a
  plan without tiers).
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


def _words(O, a, K, fl):
    out = np.zeros(K * a.n, dtype=np.float32 if fl else np.float64)
    O.lib().orc_mp_get_words(a.ptr, a.n, K, 1 if fl else 0, out.ctypes.data, a.n)
    return out.reshape(K, a.n)


def _from_words(O, w, prec):
    K, n = w.shape
    a = O.MpArray(n, prec)
    w = np.ascontiguousarray(w)
    O.lib().orc_mp_set_words(a.ptr, n, K, 1 if w.dtype == np.float32 else 0, w.ctypes.data, n)
    return a


def _slice(O, a, first, count):
    out = O.MpArray(count, a.prec)
    O.lib().orc_mp_copy(out.ptr, a.ptr + first * MPFR_T, count)
    return out


def _run_tier(M, O, tier, n, batch, seed, prec_in):
    """Inputs uniform [-1,1) at prec_in bits, split into the tier's words;
    returns (inputs as mpfr arrays, plan, x words [2][K][B][n], y words)."""
    plan = M.MultiwordPlan(n, tier)
    K, fl = plan.words, plan.word_bytes == 4
    xr, xi = O.mp_pair(n * batch, prec_in)
    O.fill_uniform(xr, xi, seed)
    x = np.stack([_words(O, xr, K, fl), _words(O, xi, K, fl)]).reshape(2, K, batch, n)
    y = np.zeros_like(x)
    plan.execute(batch, x, y)
    return xr, xi, plan, x, y


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 64, 1024, 4096, 1 << 14, 1 << 16])
def test_qd_matches_424bit_oracle(M, orc, n):
    O = orc
    batch = 2
    xr, xi, plan, x, y = _run_tier(M, O, "qd", n, batch, 70 + n, 212)
    lg = max(1, int(math.log2(n)))
    bound = math.log2(8 * lg) - 206
    for b in range(batch):
        sr, si = _slice(O, xr, b * n, n), _slice(O, xi, b * n, n)
        # the words hold the 212-bit inputs exactly: the oracle sees the same input
        gr, gi = _from_words(O, y[0, :, b], 424), _from_words(O, y[1, :, b], 424)
        dr, di = O.mp_pair(n, 424)
        if n <= 4096:
            O.mp_dft(sr, si, dr, di)
        else:
            O.MpFFT(n, 424)(sr, si, dr, di)
        e = O.mp_errors(gr, gi, dr, di)["log2_rel"]
        assert e <= bound, (n, b, e, bound)


@pytest.mark.parametrize("n", [1, 2, 4, 16, 256, 4096, 1 << 13, 1 << 16])
def test_ff_matches_96bit_oracle(M, orc, n):
    O = orc
    batch = 2
    xr, xi, plan, x, y = _run_tier(M, O, "ff", n, batch, 90 + n, 48)
    lg = max(1, int(math.log2(n)))
    bound = math.log2(8 * lg) - 44
    for b in range(batch):
        # the float pairs are the exact input of the transform
        sr, si = _from_words(O, x[0, :, b], 96), _from_words(O, x[1, :, b], 96)
        gr, gi = _from_words(O, y[0, :, b], 96), _from_words(O, y[1, :, b], 96)
        dr, di = O.mp_pair(n, 96)
        if n <= 4096:
            O.mp_dft(sr, si, dr, di)
        else:
            O.MpFFT(n, 96)(sr, si, dr, di)
        e = O.mp_errors(gr, gi, dr, di)["log2_rel"]
        assert e <= bound, (n, b, e, bound)


@pytest.mark.parametrize("tier", ["dd", "qd", "ff"])
def test_multiword_device_scaled_inverse(M, orc, tier):
    import torch

    O = orc
    n, batch = 2048, 3
    _, _, plan, x, y = _run_tier(M, O, tier, n, batch, 5, 212)
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.empty_like(d_in)
    st = torch.cuda.current_stream().cuda_stream
    plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), stream=st)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), y)
    ys = np.zeros_like(x)
    plan.execute(batch, x, ys, scaled=True)
    assert np.array_equal(ys, y / n)
    back = np.zeros_like(x)
    plan.execute(batch, ys, back, inverse=True)
    err = np.max(np.abs(back.astype(np.float64).sum(axis=1) - x.astype(np.float64).sum(axis=1)))
    assert err <= {"dd": 2.0 ** -95, "qd": 2.0 ** -50, "ff": 2.0 ** -38}[tier]


@pytest.mark.parametrize("p,form", [(24, 2), (40, 2), (41, 3), (48, 3), (53, 4), (98, 4), (106, 5), (200, 5),
                                    (201, 0)])
@pytest.mark.parametrize("n", [16, 1024])
def test_float_tier_dispatch_meets_mp_contract(M, orc, p, form, n):
    O = orc
    batch = 3
    plan = M.MpPlan(n, p, float_tiers=True)
    assert plan.form() == form
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 11 + p)
    L = O.lib()
    L.orc_mp_scale2(xr.ptr + n * MPFR_T, n, 40)  # signal 1 scaled by 2^40, signal 2 by 2^-40
    L.orc_mp_scale2(xi.ptr + n * MPFR_T, n, 40)
    L.orc_mp_scale2(xr.ptr + 2 * n * MPFR_T, n, -40)
    L.orc_mp_scale2(xi.ptr + 2 * n * MPFR_T, n, -40)
    yr, yi = O.mp_pair(n * batch, p)
    plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    for b in range(batch):
        sr, si = _slice(O, xr, b * n, n), _slice(O, xi, b * n, n)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(sr, si, dr, di)
        e = O.mp_errors(_slice(O, yr, b * n, n), _slice(O, yi, b * n, n), dr, di)["log2_rel"]
        assert e <= O.mp_bound_log2(n, p), (p, n, b, e)


def test_float_tier_out_of_window_runs_on_limbs(M, orc):
    O = orc
    n, p, batch = 64, 90, 2
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 3)
    O.lib().orc_mp_scale2(xr.ptr, n, 2000)  # beyond the double-double window
    tiers = M.MpPlan(n, p, float_tiers=True)
    limbs = M.MpPlan(n, p)
    assert tiers.form() == M.FORM_DOUBLE_DOUBLE and limbs.form() == M.FORM_LIMBS
    yr, yi = O.mp_pair(n * batch, p)
    zr, zi = O.mp_pair(n * batch, p)
    tiers.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    limbs.execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0
