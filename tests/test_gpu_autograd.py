"""GPU tests of the adjoint (MPFFT_INVERSE on the FP64 device path) and the
torch.autograd wrapper built on it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


@pytest.mark.parametrize("dims,batch", [((16,), 3), ((4096,), 2), ((1 << 16,), 1), ((8, 32), 2), ((4, 8, 16), 1)])
def test_device_inverse_matches_host_inverse_bitwise(M, dims, batch):
    """The device inverse (planes exchanged in the first and last launch) is
    bit-identical to the host path's swap(FFT(swap(x)))."""
    import torch

    n = int(np.prod(dims))
    plan = M.DPlan(n) if len(dims) == 1 else M.DPlanND(dims)
    rng = np.random.default_rng(n)
    xr, xi = rng.uniform(-1, 1, (batch, n)), rng.uniform(-1, 1, (batch, n))
    for scaled in (False, True):
        hr, hi = np.zeros_like(xr), np.zeros_like(xi)
        plan.execute(batch, xr, xi, hr, hi, scaled=scaled, inverse=True)
        d_in = torch.from_numpy(np.stack([xr, xi])).cuda()
        d_out = torch.empty_like(d_in)
        plan.execute_device(batch, d_in.data_ptr(), d_out.data_ptr(), scaled=scaled, inverse=True,
                            stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        assert np.array_equal(out[0].view(np.uint64), hr.view(np.uint64))
        assert np.array_equal(out[1].view(np.uint64), hi.view(np.uint64))


def test_autograd_gradcheck():
    """Central finite differences (torch.autograd.gradcheck, float64) for the
    forward and the inverse direction, 1-D and 2-D."""
    import torch

    from mpfft_b200.autograd import fft

    g = torch.Generator(device="cuda").manual_seed(0)
    for shape, ndim in (((2, 16), 1), ((3, 4, 8), 2)):
        z = torch.complex(torch.rand(shape, generator=g, device="cuda", dtype=torch.float64),
                          torch.rand(shape, generator=g, device="cuda", dtype=torch.float64)).requires_grad_()
        for inv in (False, True):
            assert torch.autograd.gradcheck(lambda t: fft(t, inverse=inv, ndim=ndim), (z,), eps=1e-6, atol=1e-7)


def test_autograd_weighted_power_loss():
    """loss = sum_k w_k |FFT(x)_k|^2 (w_k ~ U[0,1)): gradient = F^H (2 w y),
    against the same expression in numpy, N = 2^16, batch 4."""
    import torch

    from mpfft_b200.autograd import fft

    n, batch = 1 << 16, 4
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))
    w = rng.uniform(0, 1, n)
    xt = torch.from_numpy(x).cuda().requires_grad_()
    wt = torch.from_numpy(w).cuda()
    y = fft(xt)
    loss = (wt * (y.real ** 2 + y.imag ** 2)).sum()
    loss.backward()
    yn = np.fft.fft(x, axis=1)
    gref = np.conj(np.fft.fft(np.conj(2 * w * yn), axis=1))
    got = xt.grad.cpu().numpy()
    assert np.max(np.abs(got - gref)) <= 1e-12 * np.max(np.abs(gref))
    assert abs(loss.item() - float(np.sum(w * np.abs(yn) ** 2))) <= 1e-12 * float(np.sum(w * np.abs(yn) ** 2))


# ---------------------------------------------------------------------------
# double-double tier: the adjoint configuration (N = 2^16, batch 64)
# ---------------------------------------------------------------------------

def _split(a):
    """Dekker's splitting of float64 values into 26-bit halves (exact)."""
    c = a * 134217729.0
    hi = c - (c - a)
    return hi, a - hi


def _two_prod(a, b):
    """p + e = a * b exactly (Dekker's product, no fused multiply-add)."""
    p = a * b
    ah, al = _split(a)
    bh, bl = _split(b)
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


def _dd_weighted_cotangent(y, w):
    """2 w (y_hi + y_lo) as double-double planes, from planes (2, 2, B, n)."""
    import torch

    p, e = _two_prod(w.expand_as(y[:, 0]), y[:, 0])
    e = e + w * y[:, 1]
    s = p + e  # Fast2Sum renormalisation (|p| >= |e|)
    t = e - (s - p)
    return 2 * torch.stack((s, t), dim=1)


def test_dd_autograd_adjoint_vs_212bit_oracle(orc):
    """loss = sum_k w_k |FFT(x)_k|^2, w_k ~ U[0,1), x re/im ~ U[-1,1) at 106
    bits; N = 2^16, batch 64, double-double tier.  The gradient from
    loss.backward-style propagation (double-double cotangent 2 w y, adjoint
    kernel) is checked (a) for four signals against the reference's transform
    applied as the transpose at 212 bits, F^H g = swap(F(swap(g)))
    (lab/parallel/mp/parallel_mp_fft2.c:441-455), g = 2 w F x, and (b) for
    single components against central finite differences of the loss in
    212-bit MPFR (exact for a quadratic loss up to rounding).  Bound:
    16 log2(N) 2^-104 normwise (forward and adjoint errors add)."""
    import math

    import torch

    from mpfft_b200.autograd import dd_fft

    O = orc
    L = O.lib()
    n, batch = 1 << 16, 64
    xr, xi = O.mp_pair(n * batch, 106)
    O.fill_uniform(xr, xi, 20261205)
    planes = np.zeros((2, 2, batch, n))
    for c, a in enumerate((xr, xi)):
        L.orc_mp_get_dd(a.ptr, planes[c, 0].ctypes.data, planes[c, 1].ctypes.data, n * batch)
    w = np.random.default_rng(5).uniform(0, 1, n)
    x = torch.from_numpy(planes).cuda().requires_grad_()
    y = dd_fft(x)
    g = _dd_weighted_cotangent(y.detach(), torch.from_numpy(w).cuda())
    torch.autograd.backward(y, g)
    gx = x.grad.cpu().numpy()
    bound = math.log2(16 * 16) - 104

    def mp_of(arr2, b):  # (hi, lo) planes of signal b -> 212-bit mpfr array
        a = O.MpArray(n, 212)
        hi, lo = np.ascontiguousarray(arr2[0, b]), np.ascontiguousarray(arr2[1, b])
        L.orc_mp_set_dd(a.ptr, hi.ctypes.data, lo.ctypes.data, n)
        return a

    fft212 = O.MpFFT(n, 212)
    for b in (0, 21, 42, 63):
        sr, si = mp_of(planes[0], b), mp_of(planes[1], b)
        yr, yi = O.mp_pair(n, 212)
        fft212(sr, si, yr, yi)
        for a in (yr, yi):
            L.orc_mp_mul_d(a.ptr, w.ctypes.data, n)
            L.orc_mp_scale2(a.ptr, n, 1)
        zr, zi = O.mp_pair(n, 212)
        fft212(yi, yr, zi, zr)  # swap in, swap out: the adjoint
        gr, gi = mp_of(gx[0], b), mp_of(gx[1], b)
        e = O.mp_errors(gr, gi, zr, zi)["log2_rel"]
        assert e <= bound, (b, e, bound)
    # central differences at 212 bits, signal 0, a few components
    sr, si = mp_of(planes[0], 0), mp_of(planes[1], 0)
    gr, gi = mp_of(gx[0], 0), mp_of(gx[1], 0)
    scale = max(np.max(np.abs(gx[0, 0, 0])), np.max(np.abs(gx[1, 0, 0])))
    fd = O.MpArray(1, 212)
    diff = O.MpArray(1, 212)
    for j in (0, 1, 12345, n - 1):
        for part in (0, 1):
            L.orc_mp_power_loss_fd(fft212.ctx, w.ctypes.data, sr.ptr, si.ptr, j, part, -20, fd.ptr)
            L.orc_mp_copy(diff.ptr, (gi if part else gr).at(j), 1)
            L.orc_mp_sub_into(diff.ptr, fd.ptr)
            err = abs(diff.to_double()[0])
            assert err <= 2.0 ** bound * scale, (j, part, err, scale)
