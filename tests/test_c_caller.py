"""The boundary as a C program sees it: tests/c_caller/mpfft_caller.c is
compiled against include/mpfft_b200.h and linked to libmpfft_b200.so, and
calls mp_sr24_cp_fft / d_sr24_cp_fft the way the reference's driver does
(mpFFT.c:47-91).  On a GPU its outputs must equal the in-process calls bit for
bit and meet the oracle's bounds; without one it must fail cleanly."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cuda_available

CALLER_DIR = os.path.join(ROOT, "tests", "c_caller")
CALLER = os.path.join(CALLER_DIR, "mpfft_caller")


def _build():
    subprocess.run(["make", "-s", "-C", CALLER_DIR], check=True)
    assert os.path.exists(CALLER)


def test_c_caller_compiles_and_links():
    _build()
    if not cuda_available():
        r = subprocess.run([CALLER, "8", "64"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 2 and "mp_sr24_cp_fft: 4" in r.stderr, (r.returncode, r.stderr)


@pytest.mark.gpu
@pytest.mark.parametrize("n,p", [(1024, 256), (64, 1024)])
def test_c_caller_matches_in_process_calls_and_oracle(orc, n, p):
    import mpfft_b200 as M

    O = orc
    L = O.lib()
    if not os.path.exists(CALLER):
        _build()
    r = subprocess.run([CALLER, str(n), str(p)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    cr, ci = O.mp_pair(n, p)
    dr, di = np.zeros(n), np.zeros(n)
    for line in r.stdout.splitlines():
        kind, k, re_, im_ = line.split()
        k = int(k)
        if kind == "mp":
            assert L.orc_mp_set_str(cr.at(k), re_.encode()) == 0 and L.orc_mp_set_str(ci.at(k), im_.encode()) == 0
        else:
            dr[k], di[k] = float.fromhex(re_), float.fromhex(im_)
    # the same call in this process, on the reference's IN 2 input
    xr, xi = O.mp_pair(n, p)
    O.fill_in2(xr, xi)
    yr, yi = O.mp_pair(n, p)
    assert M.mp_sr24_cp_fft(n, 1, 0, xr.ptr, xi.ptr, yr.ptr, yi.ptr) == M.OK
    assert L.orc_mp_count_diff(cr.ptr, yr.ptr, n) == 0 and L.orc_mp_count_diff(ci.ptr, yi.ptr, n) == 0
    wr, wi = O.mp_pair(n, 2 * p)
    O.mp_dft(xr, xi, wr, wi)
    assert O.mp_errors(cr, ci, wr, wi)["log2_rel"] <= O.mp_bound_log2(n, p)
    # FP64: bit-identical to the reference's double transform (oracle restatement)
    er, ei = O.DFFT(n)(xr.to_double(), xi.to_double())
    assert np.array_equal(dr.view(np.uint64), er.view(np.uint64))
    assert np.array_equal(di.view(np.uint64), ei.view(np.uint64))
