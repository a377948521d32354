"""The oracle's FFTW stand-in against numpy / scipy (FFTW's unnormalised
definitions: REDFT10 = scipy dct type 2, REDFT01 = scipy dct type 3, r2c =
numpy rfft, c2r = numpy irfft * n)."""
import ctypes
import os

import numpy as np
import pytest
import scipy.fft

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L = ctypes.CDLL(os.path.join(ROOT, "oracle", "libsvof_oracle.so"))
L.svof_fft_plan_create.restype = ctypes.c_void_p
L.svof_fft_plan_create.argtypes = [ctypes.c_size_t]
L.svof_fft_plan_destroy.argtypes = [ctypes.c_void_p]
for fn in ("svof_dct2", "svof_dct3", "svof_fft_r2c", "svof_fft_c2r"):
    getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


@pytest.mark.parametrize("n", [2, 4, 8, 16, 128, 512, 12, 30])
def test_dct_pair(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    p = L.svof_fft_plan_create(n)
    y = np.zeros(n)
    L.svof_dct2(p, x.ctypes.data, y.ctypes.data)
    np.testing.assert_allclose(y, scipy.fft.dct(x, type=2), rtol=0, atol=1e-13 * np.abs(x).sum())
    z = np.zeros(n)
    L.svof_dct3(p, x.ctypes.data, z.ctypes.data)
    np.testing.assert_allclose(z, scipy.fft.dct(x, type=3), rtol=0, atol=1e-13 * np.abs(x).sum())
    w = np.zeros(n)
    L.svof_dct3(p, y.ctypes.data, w.ctypes.data)
    np.testing.assert_allclose(w / (2 * n), x, rtol=0, atol=1e-13)
    L.svof_fft_plan_destroy(p)


@pytest.mark.parametrize("n", [4, 8, 64, 256, 10])
def test_real_pair(n):
    rng = np.random.default_rng(100 + n)
    x = rng.standard_normal(n)
    p = L.svof_fft_plan_create(n)
    X = np.zeros(n // 2 + 1, dtype=np.complex128)
    L.svof_fft_r2c(p, x.ctypes.data, X.ctypes.data)
    np.testing.assert_allclose(X, np.fft.rfft(x), rtol=0, atol=1e-13 * np.abs(x).sum())
    # c2r ignores the imaginary parts of the DC and Nyquist terms, like FFTW
    X2 = X.copy()
    X2[0] += 5j
    if n % 2 == 0:
        X2[-1] += 7j
    y = np.zeros(n)
    L.svof_fft_c2r(p, X2.ctypes.data, y.ctypes.data)
    np.testing.assert_allclose(y, np.fft.irfft(X, n) * n, rtol=0, atol=1e-12 * np.abs(x).sum())
    L.svof_fft_plan_destroy(p)
