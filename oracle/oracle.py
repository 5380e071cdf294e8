"""ctypes bindings for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg, always as the checker.  The product library never imports it.

Two shared objects are wrapped:

* ``liboracle.so`` -- our own C restatement of the reference's hot path
  (``mpfft_oracle.c``): multiprecision and FP64 conjugate-pair split-radix
  FFTs that are bit-identical to the reference, a direct DFT at 2P bits,
  seeded input generators and error metrics.
* ``_ref/libref_*.so`` -- the reference's own FFT code files compiled
  unmodified through ``ref_shim.c`` (present where the reference tree was
  available at build time; they travel with the repository snapshot).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build(ref_root: str | None = None) -> None:
    """Compile liboracle.so and, when the reference tree exists, _ref/*.so."""
    args = ["make", "-s", "-C", HERE]
    if ref_root:
        args.append(f"REF={ref_root}")
    subprocess.run(args, check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, ul, sl, dp = C.c_void_p, C.c_ulong, C.c_long, C.POINTER(C.c_double)
    sig = {
        "orc_mp_alloc": (vp, [ul, sl]),
        "orc_mp_free": (None, [vp, ul]),
        "orc_mp_at": (vp, [vp, ul]),
        "orc_mp_set_str": (C.c_int, [vp, C.c_char_p]),
        "orc_mp_copy": (None, [vp, vp, ul]),
        "orc_mp_gather": (None, [vp, vp, ul, ul]),
        "orc_mp_set_prec_all": (None, [vp, ul, sl]),
        "orc_mp_set_d": (None, [vp, dp, ul]),
        "orc_mp_get_d": (None, [vp, dp, ul]),
        "orc_mp_set_ui": (None, [vp, ul, ul]),
        "orc_mp_scale2": (None, [vp, ul, sl]),
        "orc_mp_set_nan": (None, [vp, ul]),
        "orc_mp_set_inf": (None, [vp, ul, C.c_int]),
        "orc_mp_count_diff": (ul, [vp, vp, ul]),
        "orc_mp_to_hex": (C.c_int, [vp, C.c_char_p, C.c_int]),
        "orc_mp_from_hex": (C.c_int, [vp, C.c_char_p]),
        "orc_mp_fill_uniform": (None, [vp, vp, ul, ul]),
        "orc_mp_fill_urandom01": (None, [vp, vp, ul, ul]),
        "orc_mp_fill_in2": (None, [vp, vp, ul]),
        "orc_mp_new": (vp, [ul, sl]),
        "orc_mp_delete": (None, [vp]),
        "orc_mp_counts": (None, [vp, C.POINTER(C.c_ulong), C.c_int, C.c_int]),
        "orc_mp_fft": (None, [vp, ul, ul, sl, vp, vp, vp, vp]),
        "orc_mp_fft_top": (None, [vp, vp, vp, vp, vp]),
        "orc_mp_dft": (None, [ul, sl, vp, vp, vp, vp]),
        "orc_mp_mul_d": (None, [vp, vp, ul]),
        "orc_mp_sub_into": (None, [vp, vp]),
        "orc_mp_get_words": (None, [vp, ul, C.c_int, C.c_int, vp, ul]),
        "orc_mp_set_words": (None, [vp, ul, C.c_int, C.c_int, vp, ul]),
        "orc_mp_power_loss": (None, [vp, vp, vp, vp, vp]),
        "orc_mp_power_loss_fd": (None, [vp, vp, vp, vp, ul, C.c_int, sl, vp]),
        "orc_mp_hermitian_extend": (None, [ul, vp, vp, vp, vp]),
        "orc_mp_dft_nd": (None, [C.c_int, C.POINTER(C.c_ulong), sl, vp, vp, vp, vp]),
        "orc_mp_get_dd": (None, [vp, vp, vp, ul]),
        "orc_mp_set_dd": (None, [vp, vp, vp, ul]),
        "orc_mp_errors": (None, [ul, vp, vp, vp, vp, dp]),
        "orc_d_new": (vp, [ul]),
        "orc_d_delete": (None, [vp]),
        "orc_d_counts": (None, [vp, C.POINTER(C.c_ulong), C.c_int, C.c_int]),
        "orc_d_twiddles": (None, [vp, dp]),
        "orc_d_fft": (None, [vp, ul, ul, sl, dp, dp, dp, dp]),
        "orc_d_fft_top": (None, [vp, dp, dp, dp, dp]),
        "orc_d_fill_uniform": (None, [dp, dp, ul, ul]),
        "orc_mp_export_raw": (C.c_int, [vp, vp, ul, ul, C.c_int, vp, vp, vp]),
        "orc_mp_import_raw": (None, [vp, vp, ul, ul, C.c_int, vp, vp, vp]),
        "orc_mpfr_version": (C.c_char_p, []),
        "orc_now_ns": (C.c_ulonglong, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def dptr(a):
    """numpy float64 array -> double* (array must stay alive)."""
    return a.ctypes.data_as(C.POINTER(C.c_double))


class MpArray:
    """An owned C array of n mpfr_t elements at precision prec."""

    def __init__(self, n: int, prec: int):
        self.n, self.prec = n, prec
        self.ptr = lib().orc_mp_alloc(n, prec)

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_mp_free(self.ptr, self.n)
            self.ptr = None

    def at(self, k: int) -> int:
        return lib().orc_mp_at(self.ptr, k)

    def hex(self) -> list[str]:
        out = []
        L = lib()
        for k in range(self.n):
            need = L.orc_mp_to_hex(self.at(k), None, 0)
            buf = C.create_string_buffer(need)
            L.orc_mp_to_hex(self.at(k), buf, need)
            out.append(buf.value.decode())
        return out

    def set_hex(self, vals: list[str]) -> None:
        L = lib()
        for k, s in enumerate(vals):
            L.orc_mp_from_hex(self.at(k), s.encode())

    def to_double(self):
        import numpy as np

        v = np.zeros(self.n)
        lib().orc_mp_get_d(self.ptr, dptr(v), self.n)
        return v

    def copy_from(self, other: "MpArray") -> None:
        lib().orc_mp_copy(self.ptr, other.ptr, self.n)


def mp_pair(n: int, prec: int) -> tuple[MpArray, MpArray]:
    return MpArray(n, prec), MpArray(n, prec)


def fill_uniform(re: MpArray, im: MpArray, seed: int) -> None:
    lib().orc_mp_fill_uniform(re.ptr, im.ptr, re.n, seed)


def fill_in2(re: MpArray, im: MpArray) -> None:
    lib().orc_mp_fill_in2(re.ptr, im.ptr, re.n)


class MpFFT:
    """Our restatement of the reference mp transform for one (N, P)."""

    def __init__(self, n: int, prec: int):
        self.n, self.prec = n, prec
        self.ctx = lib().orc_mp_new(n, prec)

    def __del__(self):
        if getattr(self, "ctx", None) and _lib is not None:
            _lib.orc_mp_delete(self.ctx)
            self.ctx = None

    def __call__(self, xr, xi, yr, yi, count: bool = False):
        L = lib()
        L.orc_mp_counts(self.ctx, None, 1, 1 if count else 0)
        L.orc_mp_fft_top(self.ctx, xr.ptr, xi.ptr, yr.ptr, yi.ptr)
        if count:
            c = (C.c_ulong * 4)()
            L.orc_mp_counts(self.ctx, c, 1, 0)
            return tuple(c)
        return None


def mp_dft(xr, xi, yr, yi) -> None:
    """Direct DFT at the output arrays' precision (prec of yr[0])."""
    lib().orc_mp_dft(xr.n, yr.prec, xr.ptr, xi.ptr, yr.ptr, yi.ptr)


def mp_dft_nd(dims, xr, xi, yr, yi) -> None:
    """Row-major multi-dimensional DFT at the output arrays' precision."""
    d = (C.c_ulong * len(dims))(*dims)
    lib().orc_mp_dft_nd(len(dims), d, yr.prec, xr.ptr, xi.ptr, yr.ptr, yi.ptr)


def mp_errors(yr, yi, rr, ri) -> dict:
    """log2 normwise relative error, log2 rRMSE (re, im), log2 abs err, log2 max|ref|."""
    out = (C.c_double * 5)()
    lib().orc_mp_errors(yr.n, yr.ptr, yi.ptr, rr.ptr, ri.ptr, out)
    return {"log2_rel": out[0], "log2_rrmse_re": out[1], "log2_rrmse_im": out[2],
            "log2_abs": out[3], "log2_maxref": out[4]}


def mp_bound_log2(n: int, prec: int, c: float = 8.0) -> float:
    """log2 of the acceptance bound c*log2(N)*2^-P (log2(N) taken >= 1)."""
    return math.log2(c * max(1.0, math.log2(n))) - prec


class DFFT:
    """Our restatement of the reference FP64 transform for one N."""

    def __init__(self, n: int):
        self.n = n
        self.ctx = lib().orc_d_new(n)

    def __del__(self):
        if getattr(self, "ctx", None) and _lib is not None:
            _lib.orc_d_delete(self.ctx)
            self.ctx = None

    def __call__(self, xr, xi, count: bool = False):
        import numpy as np

        L = lib()
        yr = np.zeros(self.n)
        yi = np.zeros(self.n)
        L.orc_d_counts(self.ctx, None, 1, 1 if count else 0)
        L.orc_d_fft_top(self.ctx, dptr(xr), dptr(xi), dptr(yr), dptr(yi))
        if count:
            c = (C.c_ulong * 4)()
            L.orc_d_counts(self.ctx, c, 1, 0)
            return yr, yi, tuple(c)
        return yr, yi


def d_uniform(n: int, seed: int):
    import numpy as np

    re = np.zeros(n)
    im = np.zeros(n)
    lib().orc_d_fill_uniform(dptr(re), dptr(im), n, seed)
    return re, im


# ---------------------------------------------------------------------------
# the reference itself (compiled unmodified), one library per code file
# ---------------------------------------------------------------------------

REF_FILES = {
    "mp_par": "libref_mp_par.so",  # lab/parallel/mp/parallel_mp_fft2.c (mpFFT.c's choice, OpenMP 4 threads)
    "mp_ser": "libref_mp_ser.so",  # lab/serial/mp/serial_mp_fft3.c (fastest serial)
    "mp_v2": "libref_mp_v2.so",    # lab/serial/mp/serial_mp_fft4.c (mp_sr24_cp_fft_v2)
    "d6": "libref_d6.so",          # lab/serial/double/serial_d_fft6.c
    "d7": "libref_d7.so",          # lab/serial/double/serial_d_fft7.c (d_sr24_cp_fft_v2)
}


def ref_available(kind: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, REF_FILES[kind]))


class Ref:
    """The reference's own transform; one live instance per library per process."""

    _libs: dict = {}

    def __init__(self, kind: str, n: int, prec: int = 53):
        if kind not in Ref._libs:
            L = C.CDLL(os.path.join(REF_DIR, REF_FILES[kind]))
            L.ref_init.restype = C.c_int
            L.ref_init.argtypes = [C.c_ulong, C.c_ulong]
            L.ref_ic.argtypes = [C.c_int, C.c_ulong]
            L.ref_array.restype = C.c_void_p
            L.ref_array.argtypes = [C.c_int]
            L.ref_set_cc.argtypes = [C.c_int]
            L.ref_counts.argtypes = [C.POINTER(C.c_ulong)]
            L.ref_run.restype = C.c_ulonglong
            L.ref_run.argtypes = [C.c_ulong]
            Ref._libs[kind] = L
        self.L = Ref._libs[kind]
        self.kind, self.n, self.prec = kind, n, prec
        self.L.ref_free()
        if self.L.ref_init(n, prec) != 0:
            raise RuntimeError("reference init failed")

    def array(self, which: int) -> int:
        return self.L.ref_array(which)

    def ic(self, in_kind: int, seed: int = 0) -> None:
        self.L.ref_ic(in_kind, seed)

    def run(self, m: int = 1, count: bool = False):
        self.L.ref_set_cc(1 if count else 0)
        ns = self.L.ref_run(m)
        if count:
            c = (C.c_ulong * 4)()
            self.L.ref_counts(c)
            return ns, tuple(c)
        return ns, None

    def free(self) -> None:
        self.L.ref_free()

    # mp helpers: copy between our MpArray and the reference's arrays
    def mp_set_inputs(self, xr: MpArray, xi: MpArray) -> None:
        lib().orc_mp_copy(self.array(0), xr.ptr, self.n)
        lib().orc_mp_copy(self.array(1), xi.ptr, self.n)

    def mp_get(self, which: int, dst: MpArray) -> None:
        lib().orc_mp_copy(dst.ptr, self.array(which), self.n)

    # double helpers
    def d_view(self, which: int):
        import numpy as np

        buf = (C.c_double * self.n).from_address(self.array(which))
        return np.frombuffer(buf, dtype=np.float64, count=self.n)
