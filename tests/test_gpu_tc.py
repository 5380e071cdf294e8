"""GPU tests of the tensor-core (tcgen05 kind::i8) twiddle products used at
large precision (35..260 limbs, P from about 1050 to 8200 bits at N = 1024).

The product is checked bit for bit against its integer definition (byte
columns >= J0 of |x|*w, rounded at bit 32L-1), and the transforms that use it
against the 2P-bit MPFR DFT and against the integer-pipe streaming kernels.
"""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MPFR_T = 32


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _tc_expected(x: int, w: int, L: int) -> int:
    """sign(x) * floor((S + 2^(32L-2)) / 2^(32L-1)), S = the byte columns
    j >= J0 = (4L-8) rounded down to 16 of |x|*w."""
    j0 = (4 * L - 8) & ~15
    a = abs(x)
    full = a * w
    low = 0
    for i in range(j0):  # partial products x_i * w_c with i + c < j0
        xi = (a >> (8 * i)) & 0xFF
        if xi:
            low += (xi * (w & ((1 << (8 * (j0 - i))) - 1))) << (8 * i)
    r = (full - low + (1 << (32 * L - 2))) >> (32 * L - 1)
    return -r if x < 0 else r


def _to_planes(vals, L):
    B = len(vals)
    out = np.zeros((L, B), dtype=np.uint32)
    for b, v in enumerate(vals):
        u = v % (1 << (32 * L))
        for i in range(L):
            out[i, b] = (u >> (32 * i)) & 0xFFFFFFFF
    return out


def _from_planes(planes):
    L, B = planes.shape
    vals = []
    for b in range(B):
        u = 0
        for i in range(L):
            u |= int(planes[i, b]) << (32 * i)
        if u >> (32 * L - 1):
            u -= 1 << (32 * L)
        vals.append(u)
    return vals


@pytest.mark.parametrize("L,B", [(35, 128), (41, 77), (64, 128), (65, 1), (65, 300), (100, 129), (129, 256), (257, 130), (260, 64)])
def test_tc_product_bit_exact(M, L, B):
    import torch

    rng = random.Random(1000 * L + B)
    xs = [rng.randrange(-(1 << (32 * L - 2)) + 1, 1 << (32 * L - 2)) for _ in range(B)]
    xs[0] = (1 << (32 * L - 2)) - 1  # largest magnitude
    if B > 2:
        xs[1], xs[2] = 0, -((1 << (32 * L - 2)) - 1)
    w = rng.randrange(0, 1 << (32 * L))
    wl = np.array([(w >> (32 * i)) & 0xFFFFFFFF for i in range(L)], dtype=np.uint32)
    d_x = torch.from_numpy(_to_planes(xs, L).view(np.int32)).cuda()
    d_w = torch.from_numpy(wl.view(np.int32)).cuda()
    d_o = torch.full((L, B), 7, dtype=torch.int32, device="cuda")
    M.tc_mul(L, B, d_x.data_ptr(), d_w.data_ptr(), d_o.data_ptr())
    torch.cuda.synchronize()
    M.tc_error()
    got = _from_planes(d_o.cpu().numpy().view(np.uint32))
    for b in range(B):
        assert got[b] == _tc_expected(xs[b], w, L), b
        # within one unit of the correctly rounded full product
        full = (abs(xs[b]) * w + (1 << (32 * L - 2))) >> (32 * L - 1)
        assert abs(abs(got[b]) - full) <= 1


@pytest.mark.parametrize("n,p,batch", [(128, 1200, 40), (256, 2048, 1), (64, 2048, 130), (32, 4096, 3), (16, 8192, 2)])
def test_tc_transform_matches_oracle_and_integer_path(M, orc, n, p, batch):
    O = orc
    L = O.lib()
    tc = M.MpPlan(n, p)
    assert 35 <= tc.limbs <= 260
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 31 + p)
    yr, yi = O.mp_pair(n * batch, p)
    tc.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
    zr, zi = O.mp_pair(n * batch, p)
    M.MpPlan(n, p, tensor=False).execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
    bound = O.mp_bound_log2(n, p)
    for b in sorted({0, batch - 1}):
        sl = lambda a, pr=p: _slice(O, a, b * n, n, pr)
        sr, si = sl(xr), sl(xi)
        dr, di = O.mp_pair(n, 2 * p)
        O.mp_dft(sr, si, dr, di)
        e_tc = O.mp_errors(sl(yr), sl(yi), dr, di)["log2_rel"]
        e_int = O.mp_errors(sl(zr), sl(zi), dr, di)["log2_rel"]
        rr, ri = O.mp_pair(n, p)
        O.MpFFT(n, p)(sr, si, rr, ri)
        e_ref = O.mp_errors(rr, ri, dr, di)["log2_rel"]
        assert e_tc <= bound and e_tc <= e_ref + 0.5, (e_tc, e_ref, bound)
        assert abs(e_tc - e_int) <= 1.0, (e_tc, e_int)


def _slice(O, a, start, count, prec):
    out = O.MpArray(count, prec)
    O.lib().orc_mp_copy(out.ptr, a.ptr + start * MPFR_T, count)
    return out
