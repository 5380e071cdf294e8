"""The entry point that allocates nothing (collected last on purpose).

mpfft_mp_execute_significands_static serves callers that cannot allocate
device memory when they call -- services that reserve their whole device
memory budget at start-up, and code paths that must not pay the implicit
device-wide synchronisation of cudaMalloc/cudaFree.  Its working storage is a
static device array shared by all calls, which keeps the previous call's
contents; so the check runs two calls in a row and compares each, bit for bit
(the tolerance of the other multiprecision batch tests), with the allocating
host-array entry point mpfft_mp_execute on the same inputs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _raw_inputs(O, xr, xi, n, batch, nl):
    comp = 2 * n * batch
    mant = np.zeros(comp * nl, dtype=np.uint64)
    ex = np.zeros(comp, dtype=np.int64)
    sg = np.zeros(comp, dtype=np.uint8)
    assert O.lib().orc_mp_export_raw(xr.ptr, xi.ptr, n, batch, nl, mant.ctypes.data, ex.ctypes.data,
                                     sg.ctypes.data) == 0
    return mant, ex, sg


def test_static_scratch_entry_matches_allocating_entry(orc):
    import torch

    import mpfft_b200 as M

    O = orc
    L = O.lib()
    n, prec, batch = 256, 160, 32
    nl = (prec + 63) // 64
    plan = M.MpPlan(n, prec)
    stream = torch.cuda.current_stream()
    for call, seed in enumerate((11, 12)):
        scaled = call == 1
        xr, xi = O.mp_pair(n * batch, prec)
        O.fill_uniform(xr, xi, seed)
        if call == 1:  # different block scales and one all-zero signal on the second call
            for b in range(batch):
                for a in (xr, xi):
                    L.orc_mp_scale2(a.ptr + b * n * 32, n, (0, 40, -40)[b % 3])
            L.orc_mp_set_ui(xr.ptr + 5 * n * 32, n, 0)
            L.orc_mp_set_ui(xi.ptr + 5 * n * 32, n, 0)
        mant, ex, sg = _raw_inputs(O, xr, xi, n, batch, nl)
        d_m = torch.from_numpy(mant.view(np.int64)).cuda()
        d_e = torch.from_numpy(ex).cuda()
        d_s = torch.from_numpy(sg).cuda()
        o_m, o_e, o_s = torch.empty_like(d_m), torch.empty_like(d_e), torch.empty_like(d_s)
        plan.execute_significands_static(batch, d_m.data_ptr(), d_e.data_ptr(), d_s.data_ptr(), nl,
                                         o_m.data_ptr(), o_e.data_ptr(), o_s.data_ptr(), prec, scaled=scaled,
                                         stream=stream.cuda_stream)
        torch.cuda.synchronize()
        om = o_m.cpu().numpy().view(np.uint64).copy()
        oe = o_e.cpu().numpy().copy()
        osg = o_s.cpu().numpy().copy()
        yr, yi = O.mp_pair(n * batch, prec)
        L.orc_mp_import_raw(yr.ptr, yi.ptr, n, batch, nl, om.ctypes.data, oe.ctypes.data, osg.ctypes.data)
        zr, zi = O.mp_pair(n * batch, prec)
        plan.execute(batch, xr.ptr, xi.ptr, zr.ptr, zi.ptr, scaled=scaled)
        assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n * batch) == 0, f"call {call}"
        assert L.orc_mp_count_diff(yi.ptr, zi.ptr, n * batch) == 0, f"call {call}"

        if call == 1:
            # the defining property: a further call changes the device's free
            # memory by nothing (no allocation of any kind, cached or not)
            free0 = torch.cuda.mem_get_info()[0]
            plan.execute_significands_static(batch, d_m.data_ptr(), d_e.data_ptr(), d_s.data_ptr(), nl,
                                             o_m.data_ptr(), o_e.data_ptr(), o_s.data_ptr(), prec, scaled=scaled,
                                             stream=stream.cuda_stream)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0

    # a batch beyond the static array is rejected before any device work, also
    # where the caller's sizes would wrap a product of them
    too_big = M.lib.mpfft_static_scratch_bytes() // (16 * plan.limbs * n) + 1
    for bad in (too_big, 2**62):
        with pytest.raises(M.MpfftError) as e:
            plan.execute_significands_static(bad, 1, 1, 1, nl, 1, 1, 1, prec)
        assert e.value.code in (M.EUNSUPPORTED,)
    # only MPFFT_SCALED is accepted: an inverse request is an error, not a forward transform
    rc = M.lib.mpfft_mp_execute_significands_static(plan.h, 1, 1, 1, 1, nl, 1, 1, 1, prec, M.INVERSE, None)
    assert rc == M.EINVAL
