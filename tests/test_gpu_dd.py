"""GPU tests of the double-double tier: against a direct DFT at 212 bits
(MPFR), bound 8*log2(N)*2^-104 normwise; batches, scaling, the inverse and the
device entry point agree."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _dd_inputs(O, n, batch, seed):
    xr, xi = O.mp_pair(n * batch, 106)
    O.fill_uniform(xr, xi, seed)
    parts = []
    for a in (xr, xi):
        hi, lo = np.zeros(n * batch), np.zeros(n * batch)
        O.lib().orc_mp_get_dd(a.ptr, hi.ctypes.data, lo.ctypes.data, n * batch)
        parts.append((hi, lo))
    return xr, xi, parts[0], parts[1]


def _to_mp(O, pair, prec):
    a = O.MpArray(len(pair[0]), prec)
    O.lib().orc_mp_set_dd(a.ptr, pair[0].ctypes.data, pair[1].ctypes.data, len(pair[0]))
    return a


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 64, 1024, 2048, 4096, 16384])
def test_dd_matches_212bit_dft(M, orc, n):
    O = orc
    batch = 2
    xr, xi, pr, pi = _dd_inputs(O, n, batch, 40 + n)
    plan = M.DDPlan(n)
    yr = (np.zeros(n * batch), np.zeros(n * batch))
    yi = (np.zeros(n * batch), np.zeros(n * batch))
    plan.execute(batch, pr, pi, yr, yi)
    gr, gi = _to_mp(O, yr, 212), _to_mp(O, yi, 212)
    bound = np.log2(8 * max(1, np.log2(n))) - 104
    for b in range(batch):
        sl = lambda a: _slice(O, a, b * n, n)
        dr, di = O.mp_pair(n, 212)
        O.mp_dft(sl(xr), sl(xi), dr, di)
        e = O.mp_errors(sl(gr), sl(gi), dr, di)["log2_rel"]
        assert e <= bound, (n, b, e, bound)


def _slice(O, a, start, count):
    out = O.MpArray(count, a.prec)
    O.lib().orc_mp_copy(out.ptr, a.ptr + start * 32, count)
    return out


def test_dd_batch_scaled_inverse_device(M, orc):
    import torch

    O = orc
    n, batch = 4096, 5
    _, _, pr, pi = _dd_inputs(O, n, batch, 7)
    plan = M.DDPlan(n)
    z = lambda: (np.zeros(n * batch), np.zeros(n * batch))
    yr, yi = z(), z()
    plan.execute(batch, pr, pi, yr, yi)
    # batch = single calls
    for b in (0, batch - 1):
        s = slice(b * n, (b + 1) * n)
        sr, si = (np.zeros(n), np.zeros(n)), (np.zeros(n), np.zeros(n))
        plan.execute(1, (pr[0][s].copy(), pr[1][s].copy()), (pi[0][s].copy(), pi[1][s].copy()), sr, si)
        for got, ref in ((sr, yr), (si, yi)):
            assert np.array_equal(got[0], ref[0][s]) and np.array_equal(got[1], ref[1][s])
    # scaled = unscaled / n exactly
    ur, ui = z(), z()
    plan.execute(batch, pr, pi, ur, ui, scaled=True)
    assert np.array_equal(ur[0], yr[0] / n) and np.array_equal(ur[1], yr[1] / n)
    # inverse(scaled) of the forward returns the input within the bound
    br, bi = z(), z()
    plan.execute(batch, yr, yi, br, bi, scaled=True, inverse=True)
    err = max(np.max(np.abs((br[0] - pr[0]) + (br[1] - pr[1]))), np.max(np.abs((bi[0] - pi[0]) + (bi[1] - pi[1]))))
    assert err <= 8 * 12 * 2.0 ** -104
    # device layout [c][h][b][p], forward and inverse, bit for bit
    d_in = torch.from_numpy(np.stack([pr[0], pr[1], pi[0], pi[1]])).cuda()
    d_out = torch.empty_like(d_in)
    for inv, ref in ((False, (yr, yi)), (True, None)):
        plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), inverse=inv,
                            stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        if ref is None:
            hr, hi_ = z(), z()
            plan.execute(batch, pr, pi, hr, hi_, inverse=True)
            ref = (hr, hi_)
        assert np.array_equal(out[0], ref[0][0]) and np.array_equal(out[1], ref[0][1])
        assert np.array_equal(out[2], ref[1][0]) and np.array_equal(out[3], ref[1][1])


def _ref212_error(O, xr_pair, xi_pair, yr_pair, yi_pair, n):
    """log2 normwise error of a double-double output against the reference's
    transform run at 212 bits on the same (exactly converted) input."""
    xr, xi = _to_mp(O, xr_pair, 212), _to_mp(O, xi_pair, 212)
    gr, gi = _to_mp(O, yr_pair, 212), _to_mp(O, yi_pair, 212)
    wr, wi = O.mp_pair(n, 212)
    O.MpFFT(n, 212)(xr, xi, wr, wi)
    return O.mp_errors(gr, gi, wr, wi)["log2_rel"]


@pytest.mark.parametrize("lg", [15, 16, 17, 18, 19, 20])
def test_dd_single_signal_large_n_vs_reference_212(M, orc, lg):
    """Single signals N = 2^15 .. 2^20 (above the direct DFT's reach) against
    the reference transform at 212 bits (lab/serial/mp/serial_mp_fft3.c,
    restated bit for bit by the oracle)."""
    O = orc
    n = 1 << lg
    _, _, pr, pi = _dd_inputs(O, n, 1, 500 + lg)
    plan = M.DDPlan(n)
    yr = (np.zeros(n), np.zeros(n))
    yi = (np.zeros(n), np.zeros(n))
    plan.execute(1, pr, pi, yr, yi)
    e = _ref212_error(O, pr, pi, yr, yi, n)
    assert e <= np.log2(8 * lg) - 104, (n, e)


def test_dd_batch_4096_signals_of_4096(M, orc):
    """The batched configuration: 4096 signals of N=4096 in one call; sampled
    signals (both ends and the middle of the batch) against the reference at
    212 bits, and bit-equal to single-signal calls."""
    O = orc
    n, batch = 4096, 4096
    rng = np.random.default_rng(20261203)
    parts = []
    for _ in range(2):  # double-double inputs hi + lo with |lo| < ulp(hi)/2
        hi = rng.uniform(-1, 1, n * batch)
        parts.append((hi, hi * rng.uniform(-1, 1, n * batch) * 2.0 ** -54))
    pr, pi = parts
    plan = M.DDPlan(n)
    z = lambda: (np.zeros(n * batch), np.zeros(n * batch))
    yr, yi = z(), z()
    plan.execute(batch, pr, pi, yr, yi)
    for b in (0, 1, 2047, 2048, 4094, 4095):
        s = slice(b * n, (b + 1) * n)
        cut = lambda pair: (np.ascontiguousarray(pair[0][s]), np.ascontiguousarray(pair[1][s]))
        e = _ref212_error(O, cut(pr), cut(pi), cut(yr), cut(yi), n)
        assert e <= np.log2(8 * 12) - 104, (b, e)
    for b in (0, batch - 1):
        s = slice(b * n, (b + 1) * n)
        sr, si = (np.zeros(n), np.zeros(n)), (np.zeros(n), np.zeros(n))
        plan.execute(1, (pr[0][s].copy(), pr[1][s].copy()), (pi[0][s].copy(), pi[1][s].copy()), sr, si)
        for got, ref in ((sr, yr), (si, yi)):
            assert np.array_equal(got[0], ref[0][s]) and np.array_equal(got[1], ref[1][s])
