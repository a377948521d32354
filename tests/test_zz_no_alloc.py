"""The Poisson entry point that allocates no device memory.

svof_poisson_dct_noalloc() serves callers that cannot call cudaMalloc (a host
whose device memory belongs to a pool or budget it does not control, code that
runs where device allocation is forbidden, a plug-in that is handed only its
input and output buffers).  It keeps its spectrum and tables in a fixed
file-scope device array instead.  These tests call it through the C ABI two
times in a row (different Runge-Kutta substeps and dt) on each of several
grids -- including the grids at its size limits, whose y line solve stages
48 KB of shared memory, and a return to an earlier grid, so that the tables are
rebuilt on every change -- and check each result against the allocating entry
point svof_fluid_compute_potential_dct() on the same velocity field, within the
parity tolerance of the other tests.  The file is collected last and must pass
alone in a fresh process as well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    import simplevofsolver_b200 as svof
    fn = svof.lib().svof_poisson_dct_noalloc
    fn.argtypes = [ctypes.POINTER(svof.Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _check_grid(fn, nx, ny):
    import torch

    import simplevofsolver_b200 as svof
    from simplevofsolver_b200 import DROPLET2D_ENV, Solver, droplet2d, physical_params

    ic = droplet2d(nx, ny)
    s = Solver(ic, physical_params(DROPLET2D_ENV))
    s.run(2)  # a non-trivial velocity field
    xf = np.ascontiguousarray(ic.xf)
    shape = svof.storage_shape("psi", s.nx, s.ny)
    worst = 0.0
    for rk, dt in ((0, 1.0e-3), (2, 2.5e-3)):
        s.synchronize()
        # psi's halo corners keep the previous call's values in both paths:
        # start the output from the solver's current psi
        psi_out = torch.from_numpy(s.field("psi")).to("cuda")
        torch.cuda.synchronize()
        rc = fn(ctypes.byref(s.params), xf.ctypes.data, s.device_ptr("ux"), s.device_ptr("uy"),
                psi_out.data_ptr(), rk, dt, None)
        assert rc == 0, (nx, ny, rk)
        torch.cuda.synchronize()
        s.fluid_compute_potential_dct(rk, dt)
        ref = s.field("psi")
        got = psi_out.cpu().numpy().reshape(shape)
        rel = np.abs(got - ref).max() / np.abs(ref).max()
        assert rel <= 1e-12, (nx, ny, rk, rel)
        worst = max(worst, rel)
    s.close()
    return worst


def test_noalloc_poisson_matches_allocating_entry_point(gpu_available):
    fn = _noalloc_fn()
    _check_grid(fn, 128, 128)


@pytest.mark.parametrize("nx,ny", [(128, 512), (64, 1024), (1024, 64)])
def test_noalloc_poisson_at_its_size_limits(gpu_available, nx, ny):
    # nx * ny = 65536 (the array's capacity); 128 x 512 and 64 x 1024 stage
    # 48 KB of y lines in shared memory beside the kernel's static array
    fn = _noalloc_fn()
    _check_grid(fn, nx, ny)


def test_noalloc_tables_follow_grid_changes(gpu_available):
    # back and forth between grids: each change rebuilds and uploads the tables
    fn = _noalloc_fn()
    for nx, ny in ((128, 128), (64, 1024), (128, 128)):
        _check_grid(fn, nx, ny)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_available):
    import simplevofsolver_b200 as svof
    fn = _noalloc_fn()
    p = svof.Params(512, 256, 1.0, 0.5, 0.01, 0.01, 0.1, 0.5, 0.95, 0, 0., 0., 0., 0.)
    xf = np.linspace(0.0, 1.0, 513)
    # 512 x 256 cells exceed the 65536-cell scratch: refused before any device work
    assert fn(ctypes.byref(p), xf.ctypes.data, 1, 1, 1, 0, 1e-3, None) != 0
    # nx not a power of two: refused
    p = svof.Params(96, 64, 1.0, 1.0, 0.01, 0.01, 0.1, 0.5, 0.95, 0, 0., 0., 0., 0.)
    xf = np.linspace(0.0, 1.0, 97)
    assert fn(ctypes.byref(p), xf.ctypes.data, 1, 1, 1, 0, 1e-3, None) != 0
