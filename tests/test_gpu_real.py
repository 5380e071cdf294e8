"""GPU parity tests of the real-input (R2C) and real-output (C2R)
multiprecision transforms, through the C ABI.

The reference has no real transform (README: "only complex input"); its
complex transform of the signal with zero imaginary parts is the comparison.
Acceptance as for the complex path: normwise relative error against a direct
MPFR DFT at 2P bits <= 8*log2(N)*2^-P, and no worse than the reference's
complex transform at the same P (first N/2+1 bins).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MPFR_T = 32  # sizeof(mpfr_t) on x86-64


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _real(O, count, p, seed):
    x, junk = O.mp_pair(count, p)
    O.fill_uniform(x, junk, seed)
    return x


def _zeros(O, count, p):
    z = O.MpArray(count, p)
    O.lib().orc_mp_set_ui(z.ptr, count, 0)
    return z


def _slice(O, a, start, count, prec=None):
    out = O.MpArray(count, prec or a.prec)
    O.lib().orc_mp_copy(out.ptr, a.ptr + start * MPFR_T, count)
    return out


def _c2r_oracle(O, hr, hi, n, prec):
    """x_j = sum_k F_k exp(+2 pi i jk/n), F the Hermitian extension of the half
    spectrum, at `prec` bits: Re of the unnormalised inverse DFT, computed as
    the imaginary part of DFT(swap(F))."""
    fr, fi = O.mp_pair(n, prec)
    O.lib().orc_mp_hermitian_extend(n, hr.ptr, hi.ptr, fr.ptr, fi.ptr)
    dr, di = O.mp_pair(n, prec)
    O.mp_dft(fi, fr, dr, di)
    return di


@pytest.mark.parametrize("n,p", [(2, 64), (4, 64), (8, 64), (16, 128), (64, 256), (256, 1024), (1024, 512),
                                 (4096, 128), (1024, 1000)])
def test_r2c_matches_2p_dft_oracle(M, orc, n, p):
    O = orc
    m = n // 2
    x = _real(O, n, p, 300 + n)
    plan = M.MpRealPlan(n, p)
    yr, yi = O.mp_pair(m + 1, p)
    plan.r2c(1, x.ptr, yr.ptr, yi.ptr)
    zero = _zeros(O, n, p)
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft(x, zero, dr, di)
    hr, hi = _slice(O, dr, 0, m + 1), _slice(O, di, 0, m + 1)
    e_gpu = O.mp_errors(yr, yi, hr, hi)["log2_rel"]
    assert e_gpu <= O.mp_bound_log2(n, p), e_gpu
    # the reference's complex transform of (x, 0), same P, same bins
    rr, ri = O.mp_pair(n, p)
    O.MpFFT(n, p)(x, zero, rr, ri)
    e_ref = O.mp_errors(_slice(O, rr, 0, m + 1), _slice(O, ri, 0, m + 1), hr, hi)["log2_rel"]
    assert e_gpu <= e_ref + 0.5, (e_gpu, e_ref)
    # X_0 and X_(n/2) of a real signal are real: exactly zero imaginary parts
    v = yi.to_double()
    assert v[0] == 0.0 and v[m] == 0.0


@pytest.mark.parametrize("n,p", [(2, 64), (4, 64), (16, 128), (256, 512), (2048, 256), (1024, 1000)])
def test_c2r_matches_2p_inverse_dft_oracle(M, orc, n, p):
    """Unnormalised C2R of a random half spectrum (imaginary parts of X_0 and
    X_(n/2) set, and ignored as documented)."""
    O = orc
    m = n // 2
    hr, hi = O.mp_pair(m + 1, p)
    O.fill_uniform(hr, hi, 700 + n)
    plan = M.MpRealPlan(n, p)
    x = O.MpArray(n, p)
    plan.c2r(1, hr.ptr, hi.ptr, x.ptr)
    expect = _c2r_oracle(O, hr, hi, n, 2 * p)
    zp, z2 = _zeros(O, n, p), _zeros(O, n, 2 * p)
    e = O.mp_errors(x, zp, expect, z2)["log2_rel"]
    assert e <= O.mp_bound_log2(n, p), e


@pytest.mark.parametrize("n,p", [(8, 64), (1024, 1024), (65536, 256)])
def test_r2c_c2r_roundtrip(M, orc, n, p):
    O = orc
    m = n // 2
    x = _real(O, n, p, 11)
    plan = M.MpRealPlan(n, p)
    yr, yi = O.mp_pair(m + 1, p)
    plan.r2c(1, x.ptr, yr.ptr, yi.ptr, scaled=True)
    back = O.MpArray(n, p)
    plan.c2r(1, yr.ptr, yi.ptr, back.ptr)
    zp = _zeros(O, n, p)
    e = O.mp_errors(back, zp, x, zp)["log2_rel"]
    assert e <= O.mp_bound_log2(n, p) + 1, e


@pytest.mark.parametrize("n,p,batch", [(256, 256, 33), (64, 100, 5), (2, 64, 3)])
def test_real_batch_and_conversion_paths_agree(M, orc, n, p, batch):
    """Batched calls equal single calls, and GPU conversion equals host
    conversion, bit for bit, in both directions; signal 1 is all zeros and
    signal 2 is scaled by 2^40 (block exponents per signal)."""
    O = orc
    L = O.lib()
    m = n // 2
    x = _real(O, n * batch, p, 5)
    if batch > 1:
        L.orc_mp_set_ui(x.ptr + n * MPFR_T, n, 0)
    if batch > 2:
        L.orc_mp_scale2(x.ptr + 2 * n * MPFR_T, n, 40)
    gpu, host = M.MpRealPlan(n, p), M.MpRealPlan(n, p, host_conversion=True)
    yr, yi = O.mp_pair((m + 1) * batch, p)
    zr, zi = O.mp_pair((m + 1) * batch, p)
    gpu.r2c(batch, x.ptr, yr.ptr, yi.ptr)
    host.r2c(batch, x.ptr, zr.ptr, zi.ptr)
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, (m + 1) * batch) == 0
    assert L.orc_mp_count_diff(yi.ptr, zi.ptr, (m + 1) * batch) == 0
    for b in range(batch):
        sr, si = O.mp_pair(m + 1, p)
        gpu.r2c(1, x.ptr + b * n * MPFR_T, sr.ptr, si.ptr)
        assert L.orc_mp_count_diff(sr.ptr, yr.ptr + b * (m + 1) * MPFR_T, m + 1) == 0
        assert L.orc_mp_count_diff(si.ptr, yi.ptr + b * (m + 1) * MPFR_T, m + 1) == 0
    u, w = O.MpArray(n * batch, p), O.MpArray(n * batch, p)
    gpu.c2r(batch, yr.ptr, yi.ptr, u.ptr, scaled=True)
    host.c2r(batch, yr.ptr, yi.ptr, w.ptr, scaled=True)
    assert L.orc_mp_count_diff(u.ptr, w.ptr, n * batch) == 0
    if batch > 1:  # the zero signal stays exactly zero
        assert all(v == 0.0 for v in _slice(O, u, n, n).to_double())


def test_real_errors(M, orc):
    O = orc
    n, p = 64, 128
    plan = M.MpRealPlan(n, p)
    x = _real(O, n, p, 3)
    O.lib().orc_mp_set_nan(x.ptr, 5)
    yr, yi = O.mp_pair(n // 2 + 1, p)
    with pytest.raises(M.MpfftError) as e:
        plan.r2c(1, x.ptr, yr.ptr, yi.ptr)
    assert e.value.code == M.ENONFINITE
    cplx = M.MpPlan(n, p)
    assert M.lib.mpfft_mp_execute_r2c(cplx.h, 1, x.ptr, yr.ptr, yi.ptr, 0) == M.EINVAL
    assert M.lib.mpfft_mp_execute(plan.h, 1, x.ptr, x.ptr, yr.ptr, yi.ptr, 0) == M.EINVAL


# ---------------------------------------------------------------------------
# FP64 real transforms
# ---------------------------------------------------------------------------

def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("n", [2, 4, 8, 64, 1024, 4096, 1 << 16])
def test_d_r2c_c2r(M, orc, n):
    """Against numpy's pocketfft and against the reference's complex double
    transform (our bit-exact restatement) of the zero-imaginary signal, within
    a few units of double rounding; c2r(r2c(x)) = x."""
    O = orc
    batch, m = 3, n // 2
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, size=(batch, n))
    plan = M.DRealPlan(n)
    yr, yi = np.zeros((batch, m + 1)), np.zeros((batch, m + 1))
    plan.r2c(batch, x, yr, yi)
    tol = 8 * max(1, np.log2(n)) * 2.0 ** -53
    ref = np.fft.rfft(x, axis=1)
    assert _rel(yr + 1j * yi, ref) <= tol
    assert np.all(yi[:, 0] == 0) and np.all(yi[:, m] == 0)
    f = O.DFFT(n)
    for b in range(batch):
        cr, ci = f(x[b].copy(), np.zeros(n))
        assert _rel(yr[b] + 1j * yi[b], cr[: m + 1] + 1j * ci[: m + 1]) <= tol
    # scaled forward, unscaled inverse: the round trip
    sr, si = np.zeros_like(yr), np.zeros_like(yi)
    plan.r2c(batch, x, sr, si, scaled=True)
    back = np.zeros_like(x)
    plan.c2r(batch, sr, si, back)
    assert _rel(back, x) <= tol
    # c2r of a random half spectrum vs numpy's irfft (times n), imaginary parts of X_0, X_m ignored
    hr, hi = rng.uniform(-1, 1, size=(batch, m + 1)), rng.uniform(-1, 1, size=(batch, m + 1))
    out = np.zeros((batch, n))
    plan.c2r(batch, hr, hi, out)
    h = hr + 1j * hi
    h[:, 0] = h[:, 0].real
    h[:, m] = h[:, m].real
    assert _rel(out, np.fft.irfft(h, n=n, axis=1) * n) <= tol
    scaled = np.zeros((batch, n))
    plan.c2r(batch, hr, hi, scaled, scaled=True)
    assert np.array_equal(scaled, out / n)
