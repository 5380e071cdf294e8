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
