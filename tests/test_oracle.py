"""CPU tests that pin the oracle before anything is checked against it.

The oracle (oracle/mpfft_oracle.c) restates the reference's transforms.  It is
trusted only because these tests show it reproduces (a) the golden vectors
produced by running the reference itself (tests/golden/), (b) the reference
compiled unmodified (oracle/_ref/, where present) bit for bit, and (c) the
reference's published known answers (op counts in lab/serial/mp/OPTIONS.md:42
and lab/serial/double/OPTIONS.md:88, the IN 2 check() criterion, the
round-trip rRMSE of test()).
"""
import math

import numpy as np
import pytest

from conftest import load_golden


def _mp_from_golden(O, g):
    n, p = g["N"], g["P"]
    xr, xi = O.mp_pair(n, p)
    xr.set_hex(g["inr"])
    xi.set_hex(g["ini"])
    return xr, xi


@pytest.mark.parametrize("g", load_golden("mp_"), ids=lambda g: g["name"])
def test_mp_restatement_matches_reference_golden(orc, g):
    O = orc
    n, p = g["N"], g["P"]
    xr, xi = _mp_from_golden(O, g)
    rr, ri = O.mp_pair(n, p)
    rr.set_hex(g["outr"])
    ri.set_hex(g["outi"])
    yr, yi = O.mp_pair(n, p)
    counts = O.MpFFT(n, p)(xr, xi, yr, yi, count=True)
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, rr.ptr, n) == 0
    assert L.orc_mp_count_diff(yi.ptr, ri.ptr, n) == 0
    assert list(counts) == g["counts"]


@pytest.mark.parametrize("g", load_golden("d_"), ids=lambda g: g["name"])
def test_d_restatement_matches_reference_golden(orc, g):
    O = orc
    xr = np.array([float.fromhex(v) for v in g["inr"]])
    xi = np.array([float.fromhex(v) for v in g["ini"]])
    yr, yi, counts = O.DFFT(g["N"])(xr, xi, count=True)
    er = np.array([float.fromhex(v) for v in g["outr"]])
    ei = np.array([float.fromhex(v) for v in g["outi"]])
    assert np.array_equal(yr.view(np.uint64), er.view(np.uint64))
    assert np.array_equal(yi.view(np.uint64), ei.view(np.uint64))
    assert list(counts) == g["counts"]


def test_known_answer_op_counts(orc):
    """Op counts at N=1024 published by the reference: 3m3a 7172 mults +
    27652 adds (lab/serial/mp/OPTIONS.md:42); double CP 9668 + 25828
    (lab/serial/double/OPTIONS.md:88)."""
    O = orc
    xr, xi = O.mp_pair(1024, 64)
    O.fill_uniform(xr, xi, 1)
    yr, yi = O.mp_pair(1024, 64)
    assert O.MpFFT(1024, 64)(xr, xi, yr, yi, count=True)[:2] == (7172, 27652)
    dr, di = O.d_uniform(1024, 1)
    assert O.DFFT(1024)(dr, di, count=True)[2][:2] == (9668, 25828)


@pytest.mark.parametrize("kind", ["mp_ser", "mp_par", "mp_v2"])
@pytest.mark.parametrize("n,p", [(1, 64), (2, 64), (4, 80), (8, 100), (32, 128), (512, 320)])
def test_mp_restatement_matches_compiled_reference(orc, kind, n, p):
    O = orc
    if not O.ref_available(kind):
        pytest.skip("reference not compiled here (oracle/_ref missing)")
    ref = O.Ref(kind, n, p)
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 1000 + n + p)
    ref.mp_set_inputs(xr, xi)
    ref.run(1)
    rr, ri = O.mp_pair(n, p)
    ref.mp_get(2, rr)
    ref.mp_get(3, ri)
    ref.free()
    yr, yi = O.mp_pair(n, p)
    O.MpFFT(n, p)(xr, xi, yr, yi)
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, rr.ptr, n) == 0
    assert L.orc_mp_count_diff(yi.ptr, ri.ptr, n) == 0


@pytest.mark.parametrize("kind", ["d6", "d7"])
@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 128, 4096, 1 << 16])
def test_d_restatement_matches_compiled_reference(orc, kind, n):
    O = orc
    if not O.ref_available(kind):
        pytest.skip("reference not compiled here (oracle/_ref missing)")
    ref = O.Ref(kind, n)
    ref.ic(1, 4242 + n)
    xr, xi = ref.d_view(0).copy(), ref.d_view(1).copy()
    ref.run(1)
    er, ei = ref.d_view(2).copy(), ref.d_view(3).copy()
    ref.free()
    yr, yi = O.DFFT(n)(xr, xi)
    assert np.array_equal(yr.view(np.uint64), er.view(np.uint64))
    assert np.array_equal(yi.view(np.uint64), ei.view(np.uint64))


def test_in2_passes_reference_check_criterion(orc):
    """The reference's check(): every output component within 1e-10 of an
    O(N^2) double DFT, on the IN 2 input (parallel_mp_fft2.c:358-379)."""
    O = orc
    n, p = 1024, 1024
    xr, xi = O.mp_pair(n, p)
    O.fill_in2(xr, xi)
    yr, yi = O.mp_pair(n, p)
    O.MpFFT(n, p)(xr, xi, yr, yi)
    x = xr.to_double() + 1j * xi.to_double()
    X = np.fft.fft(x)
    assert np.max(np.abs(yr.to_double() - X.real)) < 1e-10
    assert np.max(np.abs(yi.to_double() - X.imag)) < 1e-10


@pytest.mark.parametrize("n,p", [(64, 128), (256, 256), (128, 1024)])
def test_reference_error_within_bound_of_2p_dft(orc, n, p):
    """The reference's own transform at P against the direct DFT at 2P: the
    normwise error bound c*log2(N)*2^-P (c = 8) holds for the reference."""
    O = orc
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 77 + n)
    yr, yi = O.mp_pair(n, p)
    O.MpFFT(n, p)(xr, xi, yr, yi)
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft(xr, xi, dr, di)
    e = O.mp_errors(yr, yi, dr, di)
    assert e["log2_rel"] <= O.mp_bound_log2(n, p)
    # and the oracle is not vacuous: error is well above 2^-2P
    assert e["log2_rel"] > -2 * p + 16


def test_roundtrip_swap_trick(orc):
    """The reference's test(): ifft via swap(fft(swap(X)))/N returns the input
    with rRMSE ~ 2^-P (parallel_mp_fft2.c:441-473)."""
    O = orc
    n, p = 512, 256
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 5)
    yr, yi = O.mp_pair(n, p)
    f = O.MpFFT(n, p)
    f(xr, xi, yr, yi)
    zr, zi = O.mp_pair(n, p)
    f(yi, yr, zr, zi)  # swapped inputs
    L = O.lib()
    L.orc_mp_scale2(zr.ptr, n, -9)
    L.orc_mp_scale2(zi.ptr, n, -9)
    e = O.mp_errors(zi, zr, xr, xi)  # swapped outputs vs inputs
    assert e["log2_rrmse_re"] < -p + 4 and e["log2_rrmse_im"] < -p + 4
