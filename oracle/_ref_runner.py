"""Runs the compiled reference (oracle/_ref/libsvof_ref*.so) in its own process.

TEST INFRASTRUCTURE ONLY.  Usage: _ref_runner.py LIB ICDIR NSTEPS OUT.npz NAMES [WARMUP]
The environment must hold Ra, Pr, We, coef_dt_adv, coef_dt_dif, which the
reference reads with getenv (src/config.c:14-42).  Only the integrate() calls
are timed.
"""
import ctypes
import sys
import time

import numpy as np


def main():
    lib, icdir, nsteps, out, names = sys.argv[1], sys.argv[2], int(sys.argv[3]), sys.argv[4], sys.argv[5]
    warmup = int(sys.argv[6]) if len(sys.argv) > 6 else 0
    L = ctypes.CDLL(lib)
    L.ref_init.argtypes = [ctypes.c_char_p]
    L.ref_count.argtypes = [ctypes.c_char_p]
    L.ref_count.restype = ctypes.c_long
    L.ref_get.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    L.ref_integrate.argtypes = [ctypes.c_int, ctypes.c_void_p]
    if L.ref_init(icdir.encode()) != 0:
        raise SystemExit("reference init failed")
    if warmup > 0:
        wd = np.zeros(warmup)
        if L.ref_integrate(warmup, wd.ctypes.data) != 0:
            raise SystemExit("reference integrate failed")
    dts = np.zeros(max(nsteps, 1))
    t0 = time.perf_counter()
    if L.ref_integrate(nsteps, dts.ctypes.data) != 0:
        raise SystemExit("reference integrate failed")
    seconds = time.perf_counter() - t0
    res = {"dts": dts[:nsteps], "seconds": np.array(seconds)}
    for k in [n for n in names.split(",") if n]:
        a = np.zeros(L.ref_count(k.encode()))
        L.ref_get(k.encode(), a.ctypes.data)
        res[k] = a
    np.savez(out, **res)


if __name__ == "__main__":
    main()
