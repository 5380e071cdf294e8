"""Generate golden vectors by running the REFERENCE's own FFT code.

The reference (mfrewer/mpFFT) ships no golden outputs.  This script runs its
code files -- compiled unmodified into oracle/_ref/ by oracle/Makefile -- on
fixed inputs and writes the inputs, outputs and the reference's own operation
counters as JSON fixtures next to this file.  Values are exact: mpfr numbers
as "0x<hex integer>p<exp>", doubles as float.hex().

    python tests/golden/make_golden.py      # needs oracle/_ref/*.so

Cases (small enough to commit):
  mp  : lab/serial/mp/serial_mp_fft3.c (the path mpFFT.c selects serially) and
        lab/parallel/mp/parallel_mp_fft2.c give bit-identical outputs; we
        record the serial one and check the parallel one against it here.
  d   : lab/serial/double/serial_d_fft6.c (CODE 7 is bit-identical).
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

MP_CASES = [
    # name, N, P, input kind, seed
    ("mp_n16_p64_uniform", 16, 64, "uniform", 11),
    ("mp_n64_p256_in2", 64, 256, "in2", 0),
    ("mp_n256_p256_uniform", 256, 256, "uniform", 12),
    ("mp_n1024_p64_uniform", 1024, 64, "uniform", 13),
    ("mp_n8_p100_in1", 8, 100, "ref_in1", 5),
]
D_CASES = [
    ("d_n16_in1", 16, 1, 21),
    ("d_n64_in1", 64, 1, 22),
    ("d_n1024_in1", 1024, 1, 23),
    ("d_n1024_in2", 1024, 2, 0),
]


def mp_case(name, n, p, kind, seed):
    ref = O.Ref("mp_ser", n, p)
    xr, xi = O.mp_pair(n, p)
    if kind == "uniform":
        O.fill_uniform(xr, xi, seed)
        ref.mp_set_inputs(xr, xi)
    elif kind == "in2":
        ref.ic(2)
        ref.mp_get(0, xr)
        ref.mp_get(1, xi)
    else:  # the reference's own IN 1 (seeded uniform [0,1))
        ref.ic(1, seed)
        ref.mp_get(0, xr)
        ref.mp_get(1, xi)
    _, counts = ref.run(1, count=True)
    yr, yi = O.mp_pair(n, p)
    ref.mp_get(2, yr)
    ref.mp_get(3, yi)
    ref.free()
    # the chosen parallel code must agree bit for bit
    par = O.Ref("mp_par", n, p)
    par.mp_set_inputs(xr, xi)
    par.run(1)
    zr, zi = O.mp_pair(n, p)
    par.mp_get(2, zr)
    par.mp_get(3, zi)
    par.free()
    L = O.lib()
    assert L.orc_mp_count_diff(yr.ptr, zr.ptr, n) == 0 and L.orc_mp_count_diff(yi.ptr, zi.ptr, n) == 0
    return {
        "name": name, "N": n, "P": p, "input": kind, "seed": seed,
        "source": "lab/serial/mp/serial_mp_fft3.c (== lab/parallel/mp/parallel_mp_fft2.c)",
        "counts": list(counts), "inr": xr.hex(), "ini": xi.hex(), "outr": yr.hex(), "outi": yi.hex(),
    }


def d_case(name, n, in_kind, seed):
    ref = O.Ref("d6", n)
    ref.ic(in_kind, seed)
    xr = ref.d_view(0).copy()
    xi = ref.d_view(1).copy()
    _, counts = ref.run(1, count=True)
    yr = ref.d_view(2).copy()
    yi = ref.d_view(3).copy()
    ref.free()
    return {
        "name": name, "N": n, "input": f"IN {in_kind}", "seed": seed,
        "source": "lab/serial/double/serial_d_fft6.c",
        "counts": list(counts),
        "inr": [float(v).hex() for v in xr], "ini": [float(v).hex() for v in xi],
        "outr": [float(v).hex() for v in yr], "outi": [float(v).hex() for v in yi],
    }


def main():
    for args in MP_CASES:
        d = mp_case(*args)
        with open(os.path.join(HERE, d["name"] + ".json"), "w") as f:
            json.dump(d, f)
        print("wrote", d["name"], d["counts"])
    for args in D_CASES:
        d = d_case(*args)
        with open(os.path.join(HERE, d["name"] + ".json"), "w") as f:
            json.dump(d, f)
        print("wrote", d["name"], d["counts"])


if __name__ == "__main__":
    main()
