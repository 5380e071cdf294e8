"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
validates arguments like the drop-in contract says, converts mpfr_t arrays to
device limb planes and back exactly, and fails loudly without a GPU."""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import cuda_available


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def test_library_exports_every_header_symbol(M):
    names = M.header_functions()
    assert "mp_sr24_cp_fft" in names and "d_sr24_cp_fft" in names
    for name in names:
        assert hasattr(M.lib, name), name


@pytest.mark.parametrize(
    "n,p,limbs",
    [(1, 2, 2), (2, 53, 2), (16, 64, 3), (1024, 256, 9), (1024, 1024, 33), (1 << 16, 1024, 34), (1 << 20, 512, 18)],
)
def test_limb_format(M, n, p, limbs):
    """L = ceil((P + 2 log2 N + 7)/32): sign + (log2 N + 2) headroom + at least
    P + log2 N + 4 fraction bits."""
    pl = M.MpPlan(n, p, host_only=True)
    lg = int(math.log2(n))
    assert pl.limbs == limbs
    assert pl.frac_bits == 32 * limbs - 1 - (lg + 2)
    assert pl.frac_bits >= p + lg + 4


def test_precision_beyond_supported_limbs_is_reported(M):
    assert M.MpPlan(1024, 8192, host_only=True).limbs == 257
    with pytest.raises(M.MpfftError) as e:
        M.MpPlan(1024, 20000, host_only=True)
    assert e.value.code == M.EUNSUPPORTED


@pytest.mark.parametrize("n,p", [(1, 64), (16, 64), (1024, 256), (256, 1024), (64, 53)])
def test_pack_unpack_roundtrip_exact(M, orc, n, p):
    """Inputs whose exponents lie within the fraction bits of the block scale
    survive pack -> unpack bit for bit; block exponent = max exponent."""
    O = orc
    batch = 3
    pl = M.MpPlan(n, p, host_only=True)
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 99)
    L = O.lib()
    planes = np.zeros(pl.words(batch), dtype=np.uint32)
    exps = np.zeros(batch, dtype=np.int64)
    pl.pack(batch, xr.ptr, xi.ptr, planes.ctypes.data, exps.ctypes.data)
    yr, yi = O.mp_pair(n * batch, p)
    pl.unpack(batch, planes.ctypes.data, exps.ctypes.data, yr.ptr, yi.ptr)
    assert L.orc_mp_count_diff(xr.ptr, yr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(xi.ptr, yi.ptr, n * batch) == 0
    assert np.all(exps <= 1)


def test_pack_block_scaling_and_zeros(M, orc):
    O = orc
    L = O.lib()
    n, p, batch = 64, 128, 3
    pl = M.MpPlan(n, p, host_only=True)
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 3)
    # whole signal 1 scaled up by 2^40, whole signal 2 scaled down by 2^-40
    for s, e in ((1, 40), (2, -40)):
        for arr in (xr, xi):
            sub = C.c_void_p(arr.ptr + s * n * 32)  # sizeof(mpfr_t) == 32
            L.orc_mp_scale2(sub.value, n, e)
    # signal 0 entirely zero
    L.orc_mp_set_ui(xr.ptr, n, 0)
    L.orc_mp_set_ui(xi.ptr, n, 0)
    planes = np.zeros(pl.words(batch), dtype=np.uint32)
    exps = np.zeros(batch, dtype=np.int64)
    pl.pack(batch, xr.ptr, xi.ptr, planes.ctypes.data, exps.ctypes.data)
    assert exps[0] == 0 and 40 <= exps[1] <= 41 and -40 <= exps[2] <= -39
    yr, yi = O.mp_pair(n * batch, p)
    pl.unpack(batch, planes.ctypes.data, exps.ctypes.data, yr.ptr, yi.ptr)
    assert L.orc_mp_count_diff(xr.ptr, yr.ptr, n * batch) == 0
    assert L.orc_mp_count_diff(xi.ptr, yi.ptr, n * batch) == 0


def test_pack_rejects_nonfinite(M, orc):
    O = orc
    n, p = 16, 64
    pl = M.MpPlan(n, p, host_only=True)
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 1)
    O.lib().orc_mp_set_nan(xi.ptr, 5)
    planes = np.zeros(pl.words(1), dtype=np.uint32)
    exps = np.zeros(1, dtype=np.int64)
    with pytest.raises(M.MpfftError) as e:
        pl.pack(1, xr.ptr, xi.ptr, planes.ctypes.data, exps.ctypes.data)
    assert e.value.code == M.ENONFINITE


def test_dropin_argument_validation(M, orc):
    """Invalid calls are rejected before any device work, outputs set to NaN."""
    O = orc
    xr, xi = O.mp_pair(16, 64)
    O.fill_uniform(xr, xi, 1)
    yr, yi = O.mp_pair(16, 64)
    assert M.mp_sr24_cp_fft(12, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.EINVAL
    assert M.mp_sr24_cp_fft(16, 0, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.EINVAL
    assert M.mp_sr24_cp_fft(16, 1, -1, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.EINVAL
    assert np.all(np.isnan(yr.to_double())) and np.all(np.isnan(yi.to_double()))
    assert M.mp_sr24_cp_fft_v2(16, 1, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.EINVAL
    d = np.zeros(16)
    o = np.zeros(16)
    assert M.d_sr24_cp_fft(12, 1, 0, d, d, o, o) == M.EINVAL
    assert M.d_sr24_cp_fft(16, 1, -3, d, d, o, o) == M.EINVAL
    assert np.all(np.isnan(o))
    assert M.d_sr24_cp_fft_v2(16, 2, 1, 0, d, d, o, o) == M.EINVAL


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly(M, orc):
    O = orc
    xr, xi = O.mp_pair(16, 64)
    O.fill_uniform(xr, xi, 1)
    yr, yi = O.mp_pair(16, 64)
    assert M.mp_sr24_cp_fft(16, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.ECUDA
    assert np.all(np.isnan(yr.to_double()))
    d = np.ones(16)
    o = np.zeros(16)
    assert M.d_sr24_cp_fft(16, 1, 0, d, d, o, o) == M.ECUDA
    with pytest.raises(M.MpfftError):
        M.MpPlan(16, 64)


def test_real_plan_argument_validation(M):
    """Real plans: n must be a power of two >= 2 and the format must fit the
    register kernels (checked before any device work, so no GPU is needed)."""
    for n in (0, 1, 3, 12):
        with pytest.raises(M.MpfftError) as e:
            M.MpRealPlan(n, 64)
        assert e.value.code == M.EINVAL
    with pytest.raises(M.MpfftError) as e:
        M.MpRealPlan(1024, 2048)  # 66 limbs: beyond the 34-limb register kernels
    assert e.value.code == M.EUNSUPPORTED


def test_nd_plan_argument_validation(M):
    """Rank 1..3, power-of-two dims, at most 2^26 points (mp); checked before
    any device work (a host-only mp plan needs no GPU)."""
    import ctypes as C

    pl = M.MpPlanND((16, 32), 256, host_only=True)
    lg = 9
    assert pl.n == 512 and pl.frac_bits == 32 * pl.limbs - 1 - (lg + 2)
    for dims in ((), (2, 2, 2, 2), (12, 4), (4, 0)):
        with pytest.raises(M.MpfftError) as e:
            M.MpPlanND(dims, 64, host_only=True)
        assert e.value.code == M.EINVAL
    with pytest.raises(M.MpfftError) as e:
        M.MpPlanND((1 << 14, 1 << 13), 64, host_only=True)
    assert e.value.code == M.EUNSUPPORTED
    for dims in ((3, 4), (4, 4, 4, 4)):
        d = (C.c_ulong * len(dims))(*dims)
        h = C.c_void_p()
        assert M.lib.mpfft_d_plan_create_nd(C.byref(h), len(dims), d) == M.EINVAL
