"""Failure paths that can be exercised without faulting a GPU.

* The tensor-core kernels' waits on their own MMAs are bounded.  A test-only
  setting makes every wait give up at once: the kernel then drains its MMAs,
  frees its tensor memory and returns, the call reports MPFFT_ECUDA with NaN
  outputs, and the next call with the default limit is correct again.
* MPFFT_ENOMEM: an injected failure of the next execution-buffer allocation
  (host-side fake of cudaMalloc / cudaMallocHost failing) is reported, the
  outputs are NaN, and the plan works again once the injection is off.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _check_oracle(O, xr, xi, yr, yi, n, p):
    dr, di = O.mp_pair(n, 2 * p)
    O.mp_dft(xr, xi, dr, di)
    assert O.mp_errors(yr, yi, dr, di)["log2_rel"] <= O.mp_bound_log2(n, p)


def test_tensor_core_wait_expiry_reports_error_and_recovers(M, orc):
    O = orc
    n, p = 16, 2048
    xr, xi = O.mp_pair(n, p)
    O.fill_uniform(xr, xi, 12)
    yr, yi = O.mp_pair(n, p)
    M.tc_error()  # clear any earlier flag
    M.tc_set_wait_limit(0)
    try:
        code = M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        msg = M.last_error()[1]
    finally:
        M.tc_set_wait_limit(2_000_000_000)
    assert code == M.ECUDA, msg
    assert "tensor-core wait expired" in msg
    assert np.all(np.isnan(yr.to_double())) and np.all(np.isnan(yi.to_double()))
    # the context is still usable and the next call is correct
    assert M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.OK, M.last_error()
    _check_oracle(O, xr, xi, yr, yi, n, p)


def test_injected_allocation_failure_mp_host_arrays(M, orc):
    O = orc
    n, p, batch = 64, 256, 8
    xr, xi = O.mp_pair(n * batch, p)
    O.fill_uniform(xr, xi, 5)
    yr, yi = O.mp_pair(n * batch, p)
    for host_conversion in (False, True):
        plan = M.MpPlan(n, p, host_conversion=host_conversion)  # fresh plan: no staging yet
        M.fail_allocations(0)
        try:
            with pytest.raises(M.MpfftError) as e:
                plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        finally:
            M.fail_allocations(-1)
        assert e.value.code == M.ENOMEM
        assert np.all(np.isnan(yr.to_double()))
        plan.execute(batch, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        zr, zi = O.mp_pair(n, p)
        O.lib().orc_mp_copy(zr.ptr, yr.ptr, n)
        O.lib().orc_mp_copy(zi.ptr, yi.ptr, n)
        sr, si = O.mp_pair(n, p)
        O.lib().orc_mp_copy(sr.ptr, xr.ptr, n)
        O.lib().orc_mp_copy(si.ptr, xi.ptr, n)
        _check_oracle(O, sr, si, zr, zi, n, p)


def test_injected_allocation_failure_device_scratch(M, orc):
    """Device-layout calls whose plans need scratch (a rank-2 mp plan, a
    rank-2 FP64 plan): the scratch allocation fails, then succeeds."""
    import torch

    st = torch.cuda.current_stream().cuda_stream
    mp = M.MpPlanND((8, 16), 128)
    d_in = torch.zeros(mp.words(4), dtype=torch.int32, device="cuda")
    d_out = torch.empty_like(d_in)
    dp = M.DPlanND((16, 32))
    f_in = torch.rand(2 * 4 * 512, dtype=torch.float64, device="cuda")
    f_out = torch.empty_like(f_in)
    for run in (lambda: mp.execute_device(4, d_in.data_ptr(), d_out.data_ptr(), st),
                lambda: dp.execute_device(4, f_in.data_ptr(), f_out.data_ptr(), stream=st)):
        M.fail_allocations(0)
        try:
            with pytest.raises(M.MpfftError) as e:
                run()
        finally:
            M.fail_allocations(-1)
        assert e.value.code == M.ENOMEM
        run()
    torch.cuda.synchronize()


def test_injected_allocation_failure_fp64_and_dd(M, orc):
    n, batch = 256, 3
    rng = np.random.default_rng(1)
    xr, xi = rng.uniform(-1, 1, n * batch), rng.uniform(-1, 1, n * batch)
    yr, yi = np.zeros(n * batch), np.zeros(n * batch)
    plan = M.DPlan(n)
    M.fail_allocations(0)
    try:
        with pytest.raises(M.MpfftError) as e:
            plan.execute(batch, xr, xi, yr, yi)
    finally:
        M.fail_allocations(-1)
    assert e.value.code == M.ENOMEM
    plan.execute(batch, xr, xi, yr, yi)
    ref = np.fft.fft(xr[:n] + 1j * xi[:n])
    assert np.max(np.abs(yr[:n] + 1j * yi[:n] - ref)) < 1e-12 * n
    dd = M.DDPlan(n)
    z = lambda: (np.zeros(n * batch), np.zeros(n * batch))
    ur, ui = z(), z()
    M.fail_allocations(1)  # the second allocation of the call fails
    try:
        with pytest.raises(M.MpfftError) as e:
            dd.execute(batch, (xr, 0 * xr), (xi, 0 * xi), ur, ui)
    finally:
        M.fail_allocations(-1)
    assert e.value.code == M.ENOMEM
    dd.execute(batch, (xr, 0 * xr), (xi, 0 * xi), ur, ui)
    assert np.max(np.abs(ur[0][:n] + 1j * ui[0][:n] - ref)) < 1e-12 * n
