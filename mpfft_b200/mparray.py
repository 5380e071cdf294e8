"""Owned C arrays of mpfr_t for Python callers of the drop-in entry points.

The drop-in functions take `mpfr_t *` arrays exactly like the reference
(mpFFT.h:38).  This helper allocates such arrays through the MPFR runtime
(libmpfr.so.6) and fills them with seeded uniform [-1,1) values at full
precision: one Mersenne-twister stream (gmp_randinit_mt seeded with
gmp_randseed_ui), re/im drawn interleaved per element as the reference's IN 1
does (lab/parallel/mp/parallel_mp_fft2.c:92-100), then mapped u -> 2u-1.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

MPFR_T_SIZE = 32  # sizeof(mpfr_t) on LP64: prec, sign, exp, limb pointer
_RANDSTATE_SIZE = 64  # >= sizeof(gmp_randstate_t) (32 bytes on LP64)

_mpfr = C.CDLL("libmpfr.so.6")
_gmp = C.CDLL("libgmp.so.10")

_mpfr.mpfr_init2.argtypes = [C.c_void_p, C.c_long]
_mpfr.mpfr_clear.argtypes = [C.c_void_p]
_mpfr.mpfr_urandom.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
_mpfr.mpfr_mul_2ui.argtypes = [C.c_void_p, C.c_void_p, C.c_ulong, C.c_int]
_mpfr.mpfr_sub_ui.argtypes = [C.c_void_p, C.c_void_p, C.c_ulong, C.c_int]
_mpfr.mpfr_set_ui.argtypes = [C.c_void_p, C.c_ulong, C.c_int]
_mpfr.mpfr_get_d.restype = C.c_double
_mpfr.mpfr_get_d.argtypes = [C.c_void_p, C.c_int]
_gmp.__gmp_randinit_mt.argtypes = [C.c_void_p]
_gmp.__gmp_randseed_ui.argtypes = [C.c_void_p, C.c_ulong]
_gmp.__gmp_randclear.argtypes = [C.c_void_p]


class MpfrArray:
    """n consecutive mpfr_t at precision prec, zero-initialised."""

    def __init__(self, n: int, prec: int):
        self.n, self.prec = n, prec
        self._buf = (C.c_char * (MPFR_T_SIZE * max(n, 1)))()
        self.ptr = C.addressof(self._buf)
        for k in range(n):
            _mpfr.mpfr_init2(self.ptr + k * MPFR_T_SIZE, prec)
            _mpfr.mpfr_set_ui(self.ptr + k * MPFR_T_SIZE, 0, 0)

    def at(self, k: int) -> int:
        return self.ptr + k * MPFR_T_SIZE

    def __del__(self):
        if getattr(self, "ptr", None):
            for k in range(self.n):
                _mpfr.mpfr_clear(self.ptr + k * MPFR_T_SIZE)
            self.ptr = None

    def to_double(self):
        import numpy as np

        return np.array([_mpfr.mpfr_get_d(self.at(k), 0) for k in range(self.n)])


def fill_uniform(re: MpfrArray, im: MpfrArray, seed: int) -> None:
    """re/im i.i.d. uniform [-1,1) at full precision from one seeded stream."""
    st = (C.c_char * _RANDSTATE_SIZE)()
    _gmp.__gmp_randinit_mt(st)
    _gmp.__gmp_randseed_ui(st, seed)
    for k in range(re.n):
        for a in (re, im):
            p = a.at(k)
            _mpfr.mpfr_urandom(p, st, 0)
            _mpfr.mpfr_mul_2ui(p, p, 1, 0)
            _mpfr.mpfr_sub_ui(p, p, 1, 0)
    _gmp.__gmp_randclear(st)


def synthetic_planes(n: int, limbs: int, frac_bits: int, batch: int, seed: int = 1) -> np.ndarray:
    """Limb planes [c][i][p][b] of uniform values in (-1, 1) * 2^F."""
    rng = np.random.default_rng(seed)
    words = rng.integers(0, 2**32, size=(2, limbs, n, batch), dtype=np.uint64).astype(np.uint32)
    top_bits = frac_bits - 32 * (limbs - 1)  # bits of the magnitude in the top limb
    top = words[:, limbs - 1].astype(np.int64) & ((1 << top_bits) - 1)
    neg = rng.integers(0, 2, size=top.shape, dtype=np.int64).astype(bool)
    # two's complement negation of the whole number is not needed for a valid
    # input: any integer with |A| < 2^F is valid; set the sign by the top limb
    top = np.where(neg, top - (1 << top_bits), top)
    words[:, limbs - 1] = (top & 0xFFFFFFFF).astype(np.uint32)
    return words.reshape(-1)
