"""GPU test of the uneven-batch entry point: signals of mixed lengths and
precisions (some scaled by 2^+-40) in one call give exactly the results of
single drop-in calls."""
import random

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def test_mixed_batch_equals_single_calls(M, orc):
    O = orc
    L = O.lib()
    rng = random.Random(4)
    sigs = []
    for i in range(60):
        n = rng.choice([1, 2, 16, 64, 256, 1024])
        p = rng.choice([24, 53, 106, 212, 512, 1024, 1100])
        xr, xi = O.mp_pair(n, p)
        O.fill_uniform(xr, xi, 100 + i)
        if i % 20 == 3:
            L.orc_mp_scale2(xr.ptr, n, 40)
            L.orc_mp_scale2(xi.ptr, n, 40)
        if i % 20 == 7:
            L.orc_mp_scale2(xr.ptr, n, -40)
            L.orc_mp_scale2(xi.ptr, n, -40)
        sigs.append((n, p, xr, xi, *O.mp_pair(n, p)))
    for scaled, inverse in ((False, False), (True, True)):
        M.mp_execute_mixed([s[0] for s in sigs], [s[2].ptr for s in sigs], [s[3].ptr for s in sigs],
                           [s[4].ptr for s in sigs], [s[5].ptr for s in sigs], scaled=scaled, inverse=inverse)
        fn = M.mp_sr24_cp_ifft if inverse else (M.mp_sr24_cp_fft_scaled if scaled else M.mp_sr24_cp_fft)
        for n, p, xr, xi, yr, yi in sigs:
            zr, zi = O.mp_pair(n, p)
            assert fn(n, 1, 0, xr.ptr, xi.ptr, zr.ptr, zi.ptr) == M.OK
            assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n) == 0 and L.orc_mp_count_diff(yi.ptr, zi.ptr, n) == 0, (n, p)
