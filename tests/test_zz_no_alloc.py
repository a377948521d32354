"""The Poisson entry point that allocates no device memory.

svof_poisson_dct_noalloc() serves callers that cannot call cudaMalloc (a host
whose device memory belongs to a pool or budget it does not control, code that
runs where device allocation is forbidden, a plug-in that is handed only its
input and output buffers).  It keeps its spectrum and tables in a fixed
file-scope device array instead.  This test calls it through the C ABI twice in
a row (different Runge-Kutta substeps and dt) and checks each result against
the allocating entry point svof_fluid_compute_potential_dct() on the same
velocity field, within the parity tolerance of the other tests.  It lives in a
file of its own, collected last, and must pass alone in a fresh process as
well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_poisson_matches_allocating_entry_point(gpu_available):
    import torch

    import simplevofsolver_b200 as svof
    from simplevofsolver_b200 import DROPLET2D_ENV, Solver, droplet2d, physical_params

    L = svof.lib()
    fn = L.svof_poisson_dct_noalloc
    fn.argtypes = [ctypes.POINTER(svof.Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p]
    ic = droplet2d(128, 128)
    s = Solver(ic, physical_params(DROPLET2D_ENV))
    s.run(2)  # a non-trivial velocity field
    xf = np.ascontiguousarray(ic.xf)
    shape = svof.storage_shape("psi", s.nx, s.ny)
    for rk, dt in ((0, 1.0e-3), (2, 2.5e-3)):
        s.synchronize()
        # psi's halo corners keep the previous call's values in both paths:
        # start the output from the solver's current psi
        psi_out = torch.from_numpy(s.field("psi")).to("cuda")
        torch.cuda.synchronize()
        rc = fn(ctypes.byref(s.params), xf.ctypes.data, s.device_ptr("ux"), s.device_ptr("uy"),
                psi_out.data_ptr(), rk, dt, None)
        assert rc == 0
        torch.cuda.synchronize()
        s.fluid_compute_potential_dct(rk, dt)
        ref = s.field("psi")
        got = psi_out.cpu().numpy().reshape(shape)
        rel = np.abs(got - ref).max() / np.abs(ref).max()
        assert rel <= 1e-12, rel
    s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_available):
    import simplevofsolver_b200 as svof
    L = svof.lib()
    fn = L.svof_poisson_dct_noalloc
    fn.argtypes = [ctypes.POINTER(svof.Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p]
    p = svof.Params(512, 256, 1.0, 0.5, 0.01, 0.01, 0.1, 0.5, 0.95, 0, 0., 0., 0., 0.)
    xf = np.linspace(0.0, 1.0, 513)
    # 512 x 256 cells exceed the 65536-cell scratch: refused before any device work
    assert fn(ctypes.byref(p), xf.ctypes.data, 1, 1, 1, 0, 1e-3, None) != 0
