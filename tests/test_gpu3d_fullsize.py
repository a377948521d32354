"""The 3D configurations at their full sizes, checked through properties that
do not depend on the grid size (the oracle cannot run these sizes in test
time; its parity is checked on smaller grids in test_gpu3d_parity.py):

* 256^3 FP64, 32 droplets of radii 0.04-0.08, 100 steps: the projected
  velocity is divergence-free to round-off, the flux-form vof update
  conserves the total volume to round-off, vof stays in [0, 1] up to
  round-off, and every time step is finite and positive.
* 512^3, 128 droplets of radii 0.02-0.05, 100 steps of the mixed path beside
  the FP64 path on the same GPU: velocity relative L2 error <= 1e-5 against
  the FP64 path, max |div u| <= 1e-10 and volume drift <= 1e-10; the
  pressure (modulo its mean) and vof errors are printed and bounded.
"""
import numpy as np
import pytest

from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params

pytestmark = pytest.mark.gpu

# bounds on the mixed path's pressure and vof error against the FP64 path
# (relative L2 after 100 steps at 512^3)
P_REL_L2 = 1e-4
VOF_REL_L2 = 1e-4


def volume(ic):
    return float(np.sum(ic.vof[:, :, 1:-1] * np.diff(ic.xf))) * (ic.ly / ic.ny) * (ic.lz / ic.nz)


def rel_l2(a, b):
    d = (a - b).ravel()
    return float(np.sqrt(np.dot(d, d)) / max(np.sqrt(np.dot(b.ravel(), b.ravel())), 1e-300))


def test_fp64_256_cubed_100_steps(gpu_available):
    ic = droplets3d(256, 256, 256, ndrops=32, radii=(0.04, 0.08), seed=1)
    g = Solver3D(ic, physical_params(DROPLETS3D_ENV))
    dts = g.run(100)
    assert np.all(np.isfinite(dts)) and np.all(dts > 0)
    d = g.diagnostics()
    assert d["divmax"] <= 1e-10, d
    v0 = volume(ic)
    assert abs(d["volume"] - v0) <= 1e-12 * v0, (d["volume"], v0)
    assert -1e-10 <= d["vofmin"] and d["vofmax"] <= 1 + 1e-8, d
    g.close()


def test_mixed_beside_fp64_512_cubed_100_steps(gpu_available):
    ic = droplets3d(512, 512, 512, ndrops=128, radii=(0.02, 0.05), seed=1)
    phys = physical_params(DROPLETS3D_ENV)
    f = Solver3D(ic, phys)
    m = Solver3D(ic, phys, precision="mixed")
    df_ = f.run(100)
    dm_ = m.run(100)
    assert np.all(np.isfinite(dm_)) and np.all(dm_ > 0)
    for k in ("ux", "uy", "uz"):
        err = rel_l2(m.interior(k), f.interior(k))
        assert err <= 1e-5, (k, err)
    # pressure (modulo its volume-weighted mean) and vof: stated per result
    w = np.diff(ic.xf)[None, None, :]
    errs = {}
    for k in ("p", "vof"):
        a, b = m.interior(k)[:, :, 1:-1], f.interior(k)[:, :, 1:-1]
        if k == "p":
            a = a - np.sum(a * w) / (np.sum(w) * a.shape[0] * a.shape[1])
            b = b - np.sum(b * w) / (np.sum(w) * b.shape[0] * b.shape[1])
        errs[k] = (rel_l2(a, b), float(np.abs(a - b).max() / np.abs(b).max()))
    print("mixed vs FP64 after 100 steps at 512^3 (rel L2, max rel):", errs)
    assert errs["p"][0] <= P_REL_L2 and errs["vof"][0] <= VOF_REL_L2, errs
    dm, df = m.diagnostics(), f.diagnostics()
    assert dm["divmax"] <= 1e-10 and df["divmax"] <= 1e-10, (dm, df)
    v0 = volume(ic)
    assert abs(dm["volume"] - v0) <= 1e-10 * v0, (dm["volume"], v0)
    assert abs(df["volume"] - v0) <= 1e-12 * v0, (df["volume"], v0)
    # the two paths chose nearly the same time steps
    np.testing.assert_allclose(dm_, df_, rtol=1e-5)
    m.close()
    f.close()
