"""mpfft_b200 -- B200-native conjugate-pair split-radix FFT behind mpFFT's C API.

The product is the shared library ``libmpfft_b200.so`` (sm_100a kernels plus
the C ABI declared in ``include/mpfft_b200.h``).  This module is a thin ctypes
binding to it, mirroring the reference's entry points (``mpFFT.h``):

* ``mp_sr24_cp_fft(n, s, sn, inr, ini, outr, outi)`` and friends take
  addresses of ``mpfr_t`` arrays, exactly like the C functions;
* ``MpPlan`` / ``DPlan`` expose the batched plan/execute API, including
  device-resident execution on caller-owned CUDA buffers (e.g. torch tensors).

There is no CPU fallback: if the library is missing, importing raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# MPFFT_B200_LIB may point at another build of the library (e.g. to compare builds)
LIB_PATH = os.environ.get("MPFFT_B200_LIB") or os.path.join(HERE, "libmpfft_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mpfft_b200.h")

OK, EINVAL, EUNSUPPORTED, ENONFINITE, ECUDA, ENOMEM = 0, 1, 2, 3, 4, 5
SCALED = 1
PLAN_HOST_ONLY = 2
PLAN_HOST_CONVERSION = 4
INVERSE = 8
PLAN_NO_TENSOR = 16
PLAN_TENSOR = 32
PLAN_FLOAT_TIERS = 64
PLAN_NATIVE_TIERS = 128
FORM_LIMBS, FORM_TENSOR, FORM_FLOAT_FLOAT, FORM_DOUBLE, FORM_DOUBLE_DOUBLE, FORM_QUAD_DOUBLE = range(6)


class MpfftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mpfft error {code}: {msg}")
        self.code = code


def build(verbose: bool = False) -> None:
    """Compile libmpfft_b200.so in-tree (nvcc, sm_100a)."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")], check=True, stdout=out)


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    L = C.CDLL(LIB_PATH)
    vp, ul, sl, u32p, dp = C.c_void_p, C.c_ulong, C.c_long, C.c_void_p, C.c_void_p
    sig = {
        "mp_sr24_cp_fft": (None, [ul, ul, sl, vp, vp, vp, vp]),
        "mp_sr24_cp_fft_v2": (None, [ul, ul, ul, sl, vp, vp, vp, vp]),
        "mp_sr24_cp_fft_scaled": (None, [ul, ul, sl, vp, vp, vp, vp]),
        "mp_sr24_cp_ifft": (None, [ul, ul, sl, vp, vp, vp, vp]),
        "d_sr24_cp_ifft": (None, [ul, ul, sl, dp, dp, dp, dp]),
        "d_sr24_cp_fft": (None, [ul, ul, sl, dp, dp, dp, dp]),
        "d_sr24_cp_fft_v2": (None, [ul, ul, ul, sl, dp, dp, dp, dp]),
        "d_sr24_cp_fft_scaled": (None, [ul, ul, sl, dp, dp, dp, dp]),
        "mpfft_last_error": (C.c_int, []),
        "mpfft_last_error_string": (C.c_char_p, []),
        "mpfft_mp_plan_create": (C.c_int, [C.POINTER(vp), ul, sl]),
        "mpfft_mp_plan_create_flags": (C.c_int, [C.POINTER(vp), ul, sl, C.c_uint]),
        "mpfft_mp_plan_destroy": (C.c_int, [vp]),
        "mpfft_mp_plan_limbs": (C.c_int, [vp]),
        "mpfft_mp_plan_frac_bits": (C.c_long, [vp]),
        "mpfft_mp_execute": (C.c_int, [vp, ul, vp, vp, vp, vp, C.c_uint]),
        "mpfft_mp_execute_device": (C.c_int, [vp, ul, u32p, u32p, vp]),
        "mpfft_mp_plan_create_real": (C.c_int, [C.POINTER(vp), ul, sl, C.c_uint]),
        "mpfft_mp_plan_create_nd": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(ul), sl, C.c_uint]),
        "mpfft_mp_execute_mixed": (C.c_int, [ul, C.POINTER(ul), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                             C.POINTER(vp), C.c_uint]),
        "mpfft_d_plan_create_nd": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(ul)]),
        "mpfft_d_plan_create_real": (C.c_int, [C.POINTER(vp), ul]),
        "mpfft_dd_plan_create": (C.c_int, [C.POINTER(vp), ul]),
        "mpfft_dd_execute": (C.c_int, [vp, ul, dp, dp, dp, dp, dp, dp, dp, dp, C.c_uint]),
        "mpfft_dd_execute_device": (C.c_int, [vp, ul, dp, dp, C.c_uint, vp]),
        "mpfft_d_execute_r2c": (C.c_int, [vp, ul, dp, dp, dp, C.c_uint]),
        "mpfft_d_execute_c2r": (C.c_int, [vp, ul, dp, dp, dp, C.c_uint]),
        "mpfft_mp_execute_r2c": (C.c_int, [vp, ul, vp, vp, vp, C.c_uint]),
        "mpfft_mp_execute_c2r": (C.c_int, [vp, ul, vp, vp, vp, C.c_uint]),
        "mpfft_mp_pack": (C.c_int, [vp, ul, vp, vp, u32p, vp]),
        "mpfft_mp_unpack": (C.c_int, [vp, ul, u32p, vp, vp, vp, C.c_uint]),
        "mpfft_d_plan_create": (C.c_int, [C.POINTER(vp), ul]),
        "mpfft_d_plan_destroy": (C.c_int, [vp]),
        "mpfft_d_execute": (C.c_int, [vp, ul, dp, dp, dp, dp, C.c_uint]),
        "mpfft_d_execute_device": (C.c_int, [vp, ul, dp, dp, C.c_uint, vp]),
        "mpfft_mp_plan_schedule": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
        "mpfft_mp_execute_device_timed": (C.c_int, [vp, ul, u32p, u32p, vp, C.POINTER(C.c_float)]),
        "mpfft_diag_imad_rate": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
        "mpfft_diag_tc_mul": (C.c_int, [C.c_int, ul, vp, vp, vp, vp]),
        "mpfft_diag_tc_error": (C.c_int, []),
        "mpfft_mp_execute_significands_static": (C.c_int, [vp, ul, vp, vp, vp, C.c_int, vp, vp, vp, sl, C.c_uint,
                                                           vp]),
        "mpfft_static_scratch_bytes": (C.c_size_t, []),
        "mpfft_diag_tc_set_wait_limit": (C.c_int, [C.c_ulonglong]),
        "mpfft_diag_fail_allocations": (C.c_int, [C.c_long]),
        "mpfft_mp_plan_counts": (C.c_int, [vp, C.POINTER(C.c_ulong), C.POINTER(C.c_ulong)]),
        "mpfft_mp_plan_form": (C.c_int, [vp]),
        "mpfft_diag_tc_int8_rate": (C.c_int, [C.POINTER(C.c_double)]),
        "mpfft_qd_plan_create": (C.c_int, [C.POINTER(vp), ul]),
        "mpfft_ff_plan_create": (C.c_int, [C.POINTER(vp), ul]),
        "mpfft_multiword_format": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "mpfft_multiword_execute": (C.c_int, [vp, ul, vp, vp, C.c_uint]),
        "mpfft_multiword_execute_device": (C.c_int, [vp, ul, vp, vp, C.c_uint, vp]),
        "mpfft_batch_plan_create": (C.c_int, [C.POINTER(vp), ul, C.POINTER(ul), C.POINTER(sl), C.c_uint]),
        "mpfft_batch_plan_destroy": (C.c_int, [vp]),
        "mpfft_batch_signal_format": (C.c_int, [vp, ul, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "mpfft_batch_arenas": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_size_t)]),
        "mpfft_batch_execute_device": (C.c_int, [vp, vp]),
        "mpfft_batch_execute": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.c_uint]),
        "mpfft_batch_autotune": (C.c_int, [vp, C.c_int]),
        "mpfft_batch_queue_info": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()


def header_functions() -> list[str]:
    """Names of the functions declared in include/mpfft_b200.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", src, flags=re.M)))


def last_error() -> tuple[int, str]:
    return lib.mpfft_last_error(), (lib.mpfft_last_error_string() or b"").decode()


def _check(code: int) -> None:
    if code != OK:
        raise MpfftError(code, last_error()[1])


# ---------------------------------------------------------------------------
# drop-in entry points (addresses of mpfr_t / double arrays)
# ---------------------------------------------------------------------------

def mp_sr24_cp_fft(n, s, sn, inr, ini, outr, outi) -> int:
    lib.mp_sr24_cp_fft(n, s, sn, inr, ini, outr, outi)
    return lib.mpfft_last_error()


def mp_sr24_cp_fft_v2(n, log2n, s, sn, inr, ini, outr, outi) -> int:
    lib.mp_sr24_cp_fft_v2(n, log2n, s, sn, inr, ini, outr, outi)
    return lib.mpfft_last_error()


def mp_sr24_cp_fft_scaled(n, s, sn, inr, ini, outr, outi) -> int:
    lib.mp_sr24_cp_fft_scaled(n, s, sn, inr, ini, outr, outi)
    return lib.mpfft_last_error()


def mp_sr24_cp_ifft(n, s, sn, inr, ini, outr, outi) -> int:
    lib.mp_sr24_cp_ifft(n, s, sn, inr, ini, outr, outi)
    return lib.mpfft_last_error()


def _dp(a):
    return a.ctypes.data_as(C.c_void_p) if hasattr(a, "ctypes") else a


def d_sr24_cp_fft(n, s, sn, inr, ini, outr, outi) -> int:
    lib.d_sr24_cp_fft(n, s, sn, _dp(inr), _dp(ini), _dp(outr), _dp(outi))
    return lib.mpfft_last_error()


def d_sr24_cp_fft_v2(n, log2n, s, sn, inr, ini, outr, outi) -> int:
    lib.d_sr24_cp_fft_v2(n, log2n, s, sn, _dp(inr), _dp(ini), _dp(outr), _dp(outi))
    return lib.mpfft_last_error()


def d_sr24_cp_ifft(n, s, sn, inr, ini, outr, outi) -> int:
    lib.d_sr24_cp_ifft(n, s, sn, _dp(inr), _dp(ini), _dp(outr), _dp(outi))
    return lib.mpfft_last_error()


def d_sr24_cp_fft_scaled(n, s, sn, inr, ini, outr, outi) -> int:
    lib.d_sr24_cp_fft_scaled(n, s, sn, _dp(inr), _dp(ini), _dp(outr), _dp(outi))
    return lib.mpfft_last_error()


# ---------------------------------------------------------------------------
# plans
# ---------------------------------------------------------------------------

class MpPlan:
    """Multiprecision plan for n points at `prec` bits (device limb format)."""

    def __init__(self, n: int, prec: int, host_only: bool = False, host_conversion: bool = False,
                 tensor=True, float_tiers=False):
        """tensor: True (default choice), False (integer pipes only) or
        "force" (tensor-core products from 8 limbs up).  float_tiers: True runs
        precisions a compensated floating-point tier covers within the mp
        error contract on that tier; "native" picks the smallest word format
        holding P bits."""
        h = C.c_void_p()
        flags = ((PLAN_HOST_ONLY if host_only else 0) | (PLAN_HOST_CONVERSION if host_conversion else 0)
                 | (PLAN_TENSOR if tensor == "force" else 0 if tensor else PLAN_NO_TENSOR)
                 | (PLAN_NATIVE_TIERS if float_tiers == "native" else PLAN_FLOAT_TIERS if float_tiers else 0))
        _check(lib.mpfft_mp_plan_create_flags(C.byref(h), n, prec, flags))
        self.h = h
        self.n, self.prec = n, prec
        self.limbs = lib.mpfft_mp_plan_limbs(h)
        self.frac_bits = lib.mpfft_mp_plan_frac_bits(h)

    def close(self):
        if getattr(self, "h", None):
            lib.mpfft_mp_plan_destroy(self.h)
            self.h = None

    __del__ = close

    def words(self, batch: int) -> int:
        """32-bit words of one limb-plane buffer holding `batch` signals."""
        return 2 * self.limbs * self.n * batch

    def execute(self, batch, inr, ini, outr, outi, scaled=False, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_mp_execute(self.h, batch, inr, ini, outr, outi, flags))

    def execute_device(self, batch, d_in: int, d_out: int, stream: int = 0) -> None:
        _check(lib.mpfft_mp_execute_device(self.h, batch, d_in, d_out, stream or None))

    def form(self) -> int:
        """FORM_* of the plan's host-array transforms."""
        return lib.mpfft_mp_plan_form(self.h)

    def counts(self) -> tuple[int, int]:
        """(real multiplications, real additions) of one transform, from the plan's schedule."""
        m, a = C.c_ulong(), C.c_ulong()
        _check(lib.mpfft_mp_plan_counts(self.h, C.byref(m), C.byref(a)))
        return m.value, a.value

    def schedule(self) -> list[tuple[int, int]]:
        """[(node size n, node count)] of each butterfly launch after the leaf launch."""
        a = (C.c_int * 32)()
        b = (C.c_int * 32)()
        k = lib.mpfft_mp_plan_schedule(self.h, a, b, 32)
        return [(a[i], b[i]) for i in range(max(k, 0))]

    def execute_device_timed(self, batch, d_in: int, d_out: int, stream: int = 0) -> list[float]:
        """Per-launch durations (ms): [leaf, level 0, level 1, ...]; a level
        that ran in one launch with the level before it reads 0.0."""
        nl = len(self.schedule())
        ms = (C.c_float * (nl + 1))()
        _check(lib.mpfft_mp_execute_device_timed(self.h, batch, d_in, d_out, stream or None, ms))
        return list(ms)

    def execute_significands_static(self, batch, d_mant_in, d_exp_in, d_sign_in, nl_in, d_mant_out, d_exp_out,
                                    d_sign_out, prec_out, scaled=False, stream: int = 0) -> None:
        """Device-resident MPFR fields in and out; allocates nothing (static scratch)."""
        _check(lib.mpfft_mp_execute_significands_static(self.h, batch, d_mant_in, d_exp_in, d_sign_in, nl_in,
                                                        d_mant_out, d_exp_out, d_sign_out, prec_out,
                                                        SCALED if scaled else 0, stream or None))

    def pack(self, batch, inr, ini, planes_ptr: int, exps_ptr: int) -> None:
        _check(lib.mpfft_mp_pack(self.h, batch, inr, ini, planes_ptr, exps_ptr))

    def unpack(self, batch, planes_ptr, exps_ptr, outr, outi, scaled=False) -> None:
        _check(lib.mpfft_mp_unpack(self.h, batch, planes_ptr, exps_ptr, outr, outi, SCALED if scaled else 0))


class MpPlanND(MpPlan):
    """Multiprecision multi-dimensional plan: dims (row-major, last fastest)."""

    def __init__(self, dims, prec: int, host_only: bool = False, host_conversion: bool = False,
                 tensor: bool = True):
        h = C.c_void_p()
        flags = ((PLAN_HOST_ONLY if host_only else 0) | (PLAN_HOST_CONVERSION if host_conversion else 0)
                 | (0 if tensor else PLAN_NO_TENSOR))
        d = (C.c_ulong * len(dims))(*dims)
        _check(lib.mpfft_mp_plan_create_nd(C.byref(h), len(dims), d, prec, flags))
        self.h = h
        self.dims = tuple(dims)
        self.n = 1
        for v in dims:
            self.n *= v
        self.prec = prec
        self.limbs = lib.mpfft_mp_plan_limbs(h)
        self.frac_bits = lib.mpfft_mp_plan_frac_bits(h)


class MpRealPlan:
    """Multiprecision real transform of n real points (n/2+1-point half spectrum)."""

    def __init__(self, n: int, prec: int, host_conversion: bool = False):
        h = C.c_void_p()
        _check(lib.mpfft_mp_plan_create_real(C.byref(h), n, prec, PLAN_HOST_CONVERSION if host_conversion else 0))
        self.h = h
        self.n, self.prec = n, prec
        self.limbs = lib.mpfft_mp_plan_limbs(h)
        self.frac_bits = lib.mpfft_mp_plan_frac_bits(h)

    def close(self):
        if getattr(self, "h", None):
            lib.mpfft_mp_plan_destroy(self.h)
            self.h = None

    __del__ = close

    def r2c(self, batch, x, outr, outi, scaled=False) -> None:
        _check(lib.mpfft_mp_execute_r2c(self.h, batch, x, outr, outi, SCALED if scaled else 0))

    def c2r(self, batch, inr, ini, x, scaled=False) -> None:
        _check(lib.mpfft_mp_execute_c2r(self.h, batch, inr, ini, x, SCALED if scaled else 0))


def mp_execute_mixed(ns, inr, ini, outr, outi, scaled=False, inverse=False) -> None:
    """Uneven batch: lists of lengths and of mpfr_t array addresses per signal."""
    k = len(ns)
    arr = lambda v, t: (t * k)(*v)
    flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
    _check(lib.mpfft_mp_execute_mixed(k, arr(ns, C.c_ulong), arr(inr, C.c_void_p), arr(ini, C.c_void_p),
                                      arr(outr, C.c_void_p), arr(outi, C.c_void_p), flags))


def tc_mul(limbs: int, batch: int, d_x: int, d_w: int, d_out: int, stream: int = 0) -> None:
    """Tensor-core twiddle products of `batch` operands (device limb planes)."""
    _check(lib.mpfft_diag_tc_mul(limbs, batch, d_x, d_w, d_out, stream or None))


def tc_error() -> None:
    """Raises if a bounded wait of a tensor-core kernel expired."""
    _check(lib.mpfft_diag_tc_error())


def tc_set_wait_limit(ns: int) -> None:
    """Limit of the tensor-core kernels' waits on their own MMAs (tests of the expiry path)."""
    _check(lib.mpfft_diag_tc_set_wait_limit(ns))


def fail_allocations(after: int) -> None:
    """Make the after-th execution-buffer allocation from now on (and later ones) fail; -1: off."""
    _check(lib.mpfft_diag_fail_allocations(after))


def tc_int8_rate() -> float:
    """Measured int8 tensor-core multiply-add rate of the current GPU, MAC/s."""
    v = C.c_double()
    _check(lib.mpfft_diag_tc_int8_rate(C.byref(v)))
    return v.value


def imad_rate(wide: bool = False) -> float:
    """Measured integer multiply-add rate of the current GPU, ops/s."""
    v = C.c_double()
    _check(lib.mpfft_diag_imad_rate(1 if wide else 0, C.byref(v)))
    return v.value


class DPlan:
    """FP64 plan for n points (bit-identical to the reference's double FFT)."""

    def __init__(self, n: int):
        h = C.c_void_p()
        _check(lib.mpfft_d_plan_create(C.byref(h), n))
        self.h = h
        self.n = n

    def close(self):
        if getattr(self, "h", None):
            lib.mpfft_d_plan_destroy(self.h)
            self.h = None

    __del__ = close

    def execute(self, batch, inr, ini, outr, outi, scaled=False, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_d_execute(self.h, batch, _dp(inr), _dp(ini), _dp(outr), _dp(outi), flags))

    def execute_device(self, batch, d_in: int, d_out: int, scaled=False, stream: int = 0, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_d_execute_device(self.h, batch, d_in, d_out, flags, stream or None))


class DRealPlan(DPlan):
    """FP64 real transform of n real points (n/2+1-point half spectrum)."""

    def __init__(self, n: int):
        h = C.c_void_p()
        _check(lib.mpfft_d_plan_create_real(C.byref(h), n))
        self.h = h
        self.n = n

    def r2c(self, batch, x, outr, outi, scaled=False) -> None:
        _check(lib.mpfft_d_execute_r2c(self.h, batch, _dp(x), _dp(outr), _dp(outi), SCALED if scaled else 0))

    def c2r(self, batch, inr, ini, x, scaled=False) -> None:
        _check(lib.mpfft_d_execute_c2r(self.h, batch, _dp(inr), _dp(ini), _dp(x), SCALED if scaled else 0))


class DDPlan(DPlan):
    """Double-double (about 106-bit) plan for n points."""

    def __init__(self, n: int):
        h = C.c_void_p()
        _check(lib.mpfft_dd_plan_create(C.byref(h), n))
        self.h = h
        self.n = n

    def execute(self, batch, xr, xi, yr, yi, scaled=False, inverse=False) -> None:
        """xr, xi, yr, yi: (hi, lo) pairs of float64 arrays."""
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_dd_execute(self.h, batch, _dp(xr[0]), _dp(xr[1]), _dp(xi[0]), _dp(xi[1]), _dp(yr[0]),
                                    _dp(yr[1]), _dp(yi[0]), _dp(yi[1]), flags))

    def execute_device(self, batch, d_in: int, d_out: int, scaled=False, stream: int = 0, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_dd_execute_device(self.h, batch, d_in, d_out, flags, stream or None))


class DPlanND(DPlan):
    """FP64 multi-dimensional plan: dims (row-major, last fastest)."""

    def __init__(self, dims):
        h = C.c_void_p()
        d = (C.c_ulong * len(dims))(*dims)
        _check(lib.mpfft_d_plan_create_nd(C.byref(h), len(dims), d))
        self.h = h
        self.dims = tuple(dims)
        self.n = 1
        for v in dims:
            self.n *= v


class MultiwordPlan(DPlan):
    """Compensated floating-point tier plan for n points: "dd" (double-double),
    "qd" (quad-double) or "ff" (float-float).  Arrays: numpy / device buffers in
    the layout [c][h][b][p] (c re/im, h word), float64 (float32 for "ff")."""

    def __init__(self, n: int, tier: str):
        h = C.c_void_p()
        create = {"dd": lib.mpfft_dd_plan_create, "qd": lib.mpfft_qd_plan_create, "ff": lib.mpfft_ff_plan_create}
        _check(create[tier](C.byref(h), n))
        self.h = h
        self.n, self.tier = n, tier
        k, wb = C.c_int(), C.c_int()
        _check(lib.mpfft_multiword_format(h, C.byref(k), C.byref(wb)))
        self.words, self.word_bytes = k.value, wb.value

    def execute(self, batch, x, y, scaled=False, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_multiword_execute(self.h, batch, _dp(x), _dp(y), flags))

    def execute_device(self, batch, d_in: int, d_out: int, scaled=False, stream: int = 0, inverse=False) -> None:
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_multiword_execute_device(self.h, batch, d_in, d_out, flags, stream or None))


class BatchPlan:
    """Uneven batch (lengths ns, precisions precs) as one graph launch of the
    persistent work-queue kernels; float_tiers as for MpPlan."""

    def __init__(self, ns, precs, float_tiers=False):
        k = len(ns)
        h = C.c_void_p()
        _check(lib.mpfft_batch_plan_create(C.byref(h), k, (C.c_ulong * k)(*ns), (C.c_long * k)(*precs),
                                           PLAN_NATIVE_TIERS if float_tiers == "native"
                                           else PLAN_FLOAT_TIERS if float_tiers else 0))
        self.h = h
        self.count = k

    def close(self):
        if getattr(self, "h", None):
            lib.mpfft_batch_plan_destroy(self.h)
            self.h = None

    __del__ = close

    def signal_format(self, i: int) -> tuple[int, int, int, int]:
        """(form, words or limbs, byte offset, bytes) of signal i in the arenas."""
        f, w, o, b = C.c_int(), C.c_int(), C.c_size_t(), C.c_size_t()
        _check(lib.mpfft_batch_signal_format(self.h, i, C.byref(f), C.byref(w), C.byref(o), C.byref(b)))
        return f.value, w.value, o.value, b.value

    def arenas(self) -> tuple[int, int, int]:
        a, b, n = C.c_void_p(), C.c_void_p(), C.c_size_t()
        _check(lib.mpfft_batch_arenas(self.h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value

    def execute_device(self, stream: int = 0) -> None:
        _check(lib.mpfft_batch_execute_device(self.h, stream or None))

    def execute(self, inr, ini, outr, outi, scaled=False, inverse=False) -> None:
        arr = lambda v: (C.c_void_p * self.count)(*v)
        flags = (SCALED if scaled else 0) | (INVERSE if inverse else 0)
        _check(lib.mpfft_batch_execute(self.h, arr(inr), arr(ini), arr(outr), arr(outi), flags))

    def autotune(self, save: bool = True) -> None:
        _check(lib.mpfft_batch_autotune(self.h, 1 if save else 0))

    def queues(self) -> list[dict]:
        z = C.c_int()
        nq = lib.mpfft_batch_queue_info(self.h, -1, C.byref(z), C.byref(z), C.byref(z), C.byref(z), C.byref(z))
        out = []
        for q in range(nq):
            v = [C.c_int() for _ in range(5)]
            _check(lib.mpfft_batch_queue_info(self.h, q, *[C.byref(x) for x in v]))
            out.append(dict(zip(("family", "limbs", "threads", "sub", "signals"), [x.value for x in v])))
        return out
