"""Failure detection, exercised without a GPU fault.

* Non-finite state: a NaN or an Inf placed in a host-prepared velocity
  field is met by the CFL reduction, which sets a device status word; the
  next synchronising call (svof_run, svof_fluid_decide_dt, svof_synchronize,
  their 3D forms) returns an error naming it.  The reference lets NaN pass
  silently (fmin ignores it, src/fluid/decide_dt.c:49,56).  The word is
  cleared once reported: finite fields loaded afterwards step normally.
* Out-of-memory during creation: SVOF_FAIL_ALLOC=N makes the N-th device
  buffer allocation of a creation fail (no allocation happens); every N up
  to the creation's last allocation must give an error and release what
  was allocated, and a creation without the variable still works.
* Restart files: a damaged NPY header, a wrong dtype, Fortran order or a
  shape that does not match glsizes raise ValueError naming the file (host
  only, no GPU).
* Health counters (3D): THINC intercepts whose Newton iteration missed its
  tolerance and Poisson x lines that met a pivot <= DBL_EPSILON are counted
  on the device and read with Solver3D.health; both stay 0 on the droplet
  workload in every precision, and a NaN vof cell (an interfacial cell for
  the geometry: no comparison holds for it) makes the intercept count grow.
"""
import os

import numpy as np
import pytest

from simplevofsolver_b200.workloads import (DROPLET2D_ENV, DROPLETS3D_ENV, droplet2d, droplets3d,
                                            physical_params, read_npy_dir, write_npy_dir)


# ---------------------------------------------------------------- restart files (CPU)
def test_restart_files_are_checked(tmp_path):
    ic = droplet2d(16, 8)
    d = str(tmp_path / "ok")
    write_npy_dir(ic, d)
    back = read_npy_dir(d)
    assert np.array_equal(back.fields()["vof"], ic.fields()["vof"])
    # a damaged header
    bad = str(tmp_path / "header")
    write_npy_dir(ic, bad)
    with open(os.path.join(bad, "uy.npy"), "r+b") as f:
        f.seek(0)
        f.write(b"XXXXXX")
    with pytest.raises(ValueError, match="uy.npy"):
        read_npy_dir(bad)
    # a wrong dtype
    bad = str(tmp_path / "dtype")
    write_npy_dir(ic, bad)
    np.save(os.path.join(bad, "p.npy"), ic.fields()["p"].astype(np.float32))
    with pytest.raises(ValueError, match="p.npy"):
        read_npy_dir(bad)
    # Fortran order
    bad = str(tmp_path / "order")
    write_npy_dir(ic, bad)
    np.save(os.path.join(bad, "t.npy"), np.asfortranarray(ic.fields()["t"]))
    with pytest.raises(ValueError, match="t.npy"):
        read_npy_dir(bad)
    # a shape that does not match glsizes
    bad = str(tmp_path / "shape")
    write_npy_dir(ic, bad)
    np.save(os.path.join(bad, "ux.npy"), np.zeros((8, 16)))
    with pytest.raises(ValueError, match="ux.npy"):
        read_npy_dir(bad)
    # a truncated file
    bad = str(tmp_path / "short")
    write_npy_dir(ic, bad)
    with open(os.path.join(bad, "vof.npy"), "r+b") as f:
        f.truncate(100)
    with pytest.raises(ValueError, match="vof.npy"):
        read_npy_dir(bad)


def test_restart_files_are_checked_3d(tmp_path):
    ic = droplets3d(16, 16, 8, ndrops=1, radii=(0.1, 0.15))
    d = str(tmp_path / "ok3")
    write_npy_dir(ic, d)
    read_npy_dir(d)
    np.save(os.path.join(d, "uz.npy"), np.zeros((8, 16, 17)))
    with pytest.raises(ValueError, match="uz.npy"):
        read_npy_dir(d)


# ---------------------------------------------------------------- non-finite state (GPU)
@pytest.mark.gpu
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_velocity_is_reported_2d(gpu_available, bad):
    from simplevofsolver_b200 import Solver, SvofError
    ic = droplet2d(32, 32)
    s = Solver(ic, physical_params(DROPLET2D_ENV))
    s.run(1)
    ux = s.interior("ux")
    ux[7, 5] = bad
    s.load_interior("ux", ux)
    with pytest.raises(SvofError, match="non-finite"):
        s.run(1)
    # cleared once reported: finite fields step again
    for k, v in ic.fields().items():
        s.load_interior(k, v)
    s.run(2)
    s.close()


@pytest.mark.gpu
def test_non_finite_velocity_is_reported_by_decide_dt(gpu_available):
    from simplevofsolver_b200 import Solver, SvofError
    ic = droplet2d(32, 32)
    s = Solver(ic, physical_params(DROPLET2D_ENV))
    uy = s.interior("uy")
    uy[3, 9] = np.nan
    s.load_interior("uy", uy)
    with pytest.raises(SvofError, match="non-finite"):
        s.fluid_decide_dt()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ux", "uz"])
def test_non_finite_velocity_is_reported_3d(gpu_available, name):
    from simplevofsolver_b200 import Solver3D, SvofError
    ic = droplets3d(32, 16, 16, ndrops=2, radii=(0.1, 0.2))
    s = Solver3D(ic, physical_params(DROPLETS3D_ENV))
    s.run(1)
    a = s.field(name)
    a[5, 6, 7] = np.nan
    s.set_field(name, a)
    with pytest.raises(SvofError, match="non-finite"):
        s.run(1)
    for k, v in ic.fields().items():
        s.load_interior(k, v)
    s.run(1)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_dc"])
def test_health_counters_3d(gpu_available, precision):
    from simplevofsolver_b200 import Solver3D
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    s = Solver3D(ic, physical_params(DROPLETS3D_ENV), precision=precision)
    s.run(5)
    assert s.health() == {"newton_unconverged": 0, "small_pivots": 0}
    v = s.field("vof")
    v[8, 8, 12] = np.nan
    s.set_field("vof", v)
    s.interface_compute_curvature_tensor()
    h = s.health(reset=True)
    assert h["newton_unconverged"] >= 1 and h["small_pivots"] == 0, h
    assert s.health() == {"newton_unconverged": 0, "small_pivots": 0}
    for k, a in ic.fields().items():
        s.load_interior(k, a)
    s.run(2)
    assert s.health() == {"newton_unconverged": 0, "small_pivots": 0}


# ---------------------------------------------------------------- allocation failure (GPU)
def _sweep_alloc_failures(make):
    """creations with SVOF_FAIL_ALLOC = 1, 2, ... until one succeeds: each
    earlier one must fail with an error; returns the number of allocations"""
    from simplevofsolver_b200 import SvofError
    import torch
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    n = 0
    try:
        for n in range(1, 400):
            os.environ["SVOF_FAIL_ALLOC"] = str(n)
            try:
                s = make()
            except SvofError:
                continue
            s.close()
            break
        else:
            raise AssertionError("a creation never succeeded")
    finally:
        os.environ.pop("SVOF_FAIL_ALLOC", None)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    # the failed creations released their buffers (a few MB of slack for
    # the driver's own bookkeeping)
    assert free0 - free1 < 64 << 20, (free0, free1)
    s = make()
    s.close()
    return n


@pytest.mark.gpu
def test_allocation_failures_during_creation_2d(gpu_available):
    from simplevofsolver_b200 import Solver
    ic = droplet2d(64, 64)
    n = _sweep_alloc_failures(lambda: Solver(ic, physical_params(DROPLET2D_ENV)))
    assert n > 10


@pytest.mark.gpu
def test_allocation_failures_during_creation_3d(gpu_available):
    from simplevofsolver_b200 import Solver3D
    ic = droplets3d(32, 16, 16, ndrops=2, radii=(0.1, 0.2))
    n = _sweep_alloc_failures(lambda: Solver3D(ic, physical_params(DROPLETS3D_ENV)))
    assert n > 10
