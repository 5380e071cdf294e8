"""GPU tests of uneven batches as one graph launch of the persistent
work-queue kernels (the configuration with N log-uniform over 2^4..2^16 and
precisions drawn from {24, 53, 106, 212, 512, 1024}, 5 % of the signals
scaled by 2^+-40; here with N up to 2^11 so the oracle finishes in seconds).

Every output equals the single call of the same signal (an mp plan with the
same tier flags, one signal) bit for bit, and the single calls meet their
error bounds against the 2P-bit oracle: the multiprecision contract
8 log2(N) 2^-P for limbs, the tier's own bound for the native floating tiers.
"""
import ctypes as C
import glob
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECS = (24, 53, 106, 212, 512, 1024)
TIER_BITS = {2: 44, 3: 50, 4: 101, 5: 206}  # form -> log2 bound exponent of the tier's own error


def _cudart():
    """The CUDA runtime library (for plain device-to-host copies of the arenas)."""
    try:
        return C.CDLL("libcudart.so.12")
    except OSError:
        import torch

        d = os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib")
        return C.CDLL(sorted(glob.glob(os.path.join(d, "libcudart.so*")))[0])


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def _batch(O, count, seed, lg_max):
    rng = np.random.default_rng(seed)
    lgs = rng.integers(4, lg_max + 1, count)
    precs = rng.choice(PRECS, count)
    scales = rng.choice([0, 40, -40], count, p=[0.9, 0.05, 0.05])
    sig = []
    for i in range(count):
        n, p = 1 << int(lgs[i]), int(precs[i])
        xr, xi = O.mp_pair(n, p)
        O.fill_uniform(xr, xi, seed * 1000 + i)
        if scales[i]:
            O.lib().orc_mp_scale2(xr.ptr, n, int(scales[i]))
            O.lib().orc_mp_scale2(xi.ptr, n, int(scales[i]))
        sig.append((n, p, xr, xi))
    return sig


@pytest.mark.parametrize("tiers", ["native", True, False])
def test_queue_batch_equals_single_calls(M, orc, tiers):
    O = orc
    L = O.lib()
    sig = _batch(O, 90, 7, 11)
    plan = M.BatchPlan([s[0] for s in sig], [s[1] for s in sig], float_tiers=tiers)
    outs = [O.mp_pair(n, p) for n, p, _, _ in sig]
    plan.execute([s[2].ptr for s in sig], [s[3].ptr for s in sig], [o[0].ptr for o in outs],
                 [o[1].ptr for o in outs])
    forms = set()
    for i, (n, p, xr, xi) in enumerate(sig):
        form = plan.signal_format(i)[0]
        forms.add(form)
        single = M.MpPlan(n, p, float_tiers=tiers)
        assert single.form() == form, (i, n, p)
        zr, zi = O.mp_pair(n, p)
        single.execute(1, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
        assert L.orc_mp_count_diff(zr.ptr, outs[i][0].ptr, n) == 0, (i, n, p, form)
        assert L.orc_mp_count_diff(zi.ptr, outs[i][1].ptr, n) == 0, (i, n, p, form)
        if i % 6 == 0:  # the single call against the 2P-bit DFT
            dr, di = O.mp_pair(n, 2 * p)
            O.mp_dft(xr, xi, dr, di)
            e = O.mp_errors(zr, zi, dr, di)["log2_rel"]
            lg = max(1, int(math.log2(n)))
            bound = O.mp_bound_log2(n, p)
            if tiers == "native" and form > 1:  # the tier's own error, or the rounding to P bits
                bound = max(bound, math.log2(8 * lg) - TIER_BITS[form])
            assert e <= bound, (i, n, p, form, e, bound)
    if tiers == "native":
        assert forms == {0, 2, 3, 4, 5}
    elif tiers is False:
        assert forms == {0}


def test_queue_device_arena_scaled_inverse_and_autotune(M, orc, tmp_path, monkeypatch):
    """The device entry runs the same graph; scaled / inverse host calls; the
    autotuner's choices change no result and are written to the tune file."""
    import torch

    O = orc
    L = O.lib()
    monkeypatch.setenv("MPFFT_AUTOTUNE_FILE", str(tmp_path / "tune.json"))
    sig = _batch(O, 40, 11, 10)
    ns, ps = [s[0] for s in sig], [s[1] for s in sig]
    plan = M.BatchPlan(ns, ps, float_tiers="native")
    outs = [O.mp_pair(n, p) for n, p in zip(ns, ps)]
    ins = ([s[2].ptr for s in sig], [s[3].ptr for s in sig])
    plan.execute(*ins, [o[0].ptr for o in outs], [o[1].ptr for o in outs])
    d_in, d_out, nbytes = plan.arenas()
    rt = _cudart()
    before, after = np.zeros(nbytes, np.uint8), np.ones(nbytes, np.uint8)
    # the device entry on the arena the host call staged gives the same output arena
    assert rt.cudaMemcpy(C.c_void_p(before.ctypes.data), C.c_void_p(d_out), C.c_size_t(nbytes), 2) == 0
    plan.execute_device(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rt.cudaMemcpy(C.c_void_p(after.ctypes.data), C.c_void_p(d_out), C.c_size_t(nbytes), 2) == 0
    assert np.array_equal(before, after)
    plan.autotune(save=True)
    assert (tmp_path / "tune.json").exists()
    outs2 = [O.mp_pair(n, p) for n, p in zip(ns, ps)]
    plan.execute(*ins, [o[0].ptr for o in outs2], [o[1].ptr for o in outs2])
    for (n, p), a, b in zip(zip(ns, ps), outs, outs2):
        assert L.orc_mp_count_diff(a[0].ptr, b[0].ptr, n) == 0 and L.orc_mp_count_diff(a[1].ptr, b[1].ptr, n) == 0
    # a new plan for the same batch reads the tuned shapes
    again = M.BatchPlan(ns, ps, float_tiers="native")
    assert again.queues() == plan.queues()
    # scaled = unscaled x 2^-log2 N exactly; inverse = swap(forward(swap))
    outs3 = [O.mp_pair(n, p) for n, p in zip(ns, ps)]
    plan.execute(*ins, [o[0].ptr for o in outs3], [o[1].ptr for o in outs3], scaled=True)
    for (n, p), a, b in zip(zip(ns, ps), outs, outs3):
        for k in (0, 1):
            L.orc_mp_scale2(a[k].ptr, n, -int(math.log2(n)))
            assert L.orc_mp_count_diff(a[k].ptr, b[k].ptr, n) == 0
    outs4 = [O.mp_pair(n, p) for n, p in zip(ns, ps)]
    plan.execute(*ins, [o[0].ptr for o in outs4], [o[1].ptr for o in outs4], inverse=True)
    outs5 = [O.mp_pair(n, p) for n, p in zip(ns, ps)]
    plan.execute(ins[1], ins[0], [o[1].ptr for o in outs5], [o[0].ptr for o in outs5])
    for (n, p), a, b in zip(zip(ns, ps), outs4, outs5):
        assert L.orc_mp_count_diff(a[0].ptr, b[0].ptr, n) == 0 and L.orc_mp_count_diff(a[1].ptr, b[1].ptr, n) == 0


def test_queue_long_limb_signals_run_as_groups(M, orc):
    """Limb signals of 4096 points and more run as groups (per-level launches
    over every signal of one (N, L)) instead of in their queue; their outputs
    equal the single calls bit for bit, next to short signals of the same
    limb counts in the queues, and the plan reports each group (threads 0,
    sub = its length)."""
    O = orc
    L = O.lib()
    spec = [(4096, 1024), (8192, 1024), (4096, 1024), (16384, 512), (4096, 100), (8192, 512),
            (256, 1024), (1024, 512), (64, 100), (4096, 53)]
    sig = []
    for i, (n, p) in enumerate(spec):
        xr, xi = O.mp_pair(n, p)
        O.fill_uniform(xr, xi, 500 + i)
        if i == 2:
            L.orc_mp_scale2(xr.ptr, n, 40)
            L.orc_mp_scale2(xi.ptr, n, 40)
        sig.append((n, p, xr, xi))
    plan = M.BatchPlan([s[0] for s in sig], [s[1] for s in sig], float_tiers=False)
    groups = [q for q in plan.queues() if q["threads"] == 0]
    assert sorted((q["sub"], q["signals"]) for q in groups) == [(4096, 1), (4096, 1), (4096, 2), (8192, 1),
                                                                 (8192, 1), (16384, 1)], plan.queues()
    outs = [O.mp_pair(n, p) for n, p, _, _ in sig]
    plan.execute([s[2].ptr for s in sig], [s[3].ptr for s in sig], [o[0].ptr for o in outs],
                 [o[1].ptr for o in outs])
    for i, (n, p, xr, xi) in enumerate(sig):
        single = M.MpPlan(n, p, float_tiers=False)
        zr, zi = O.mp_pair(n, p)
        single.execute(1, xr.ptr, xi.ptr, zr.ptr, zi.ptr)
        assert L.orc_mp_count_diff(zr.ptr, outs[i][0].ptr, n) == 0, (i, n, p)
        assert L.orc_mp_count_diff(zi.ptr, outs[i][1].ptr, n) == 0, (i, n, p)
    # one grouped signal against the reference's transform at 2P bits
    n, p, xr, xi = sig[0]
    wr, wi = O.mp_pair(n, 2 * p)
    O.MpFFT(n, 2 * p)(xr, xi, wr, wi)
    e = O.mp_errors(outs[0][0], outs[0][1], wr, wi)["log2_rel"]
    assert e <= O.mp_bound_log2(n, p), (e, O.mp_bound_log2(n, p))
