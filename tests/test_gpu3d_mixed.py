"""The mixed-precision 3D path (SVOF3_MIXED) against the FP64 oracle and the
FP64 GPU path.

The mixed path keeps the state (velocities, pressure, psi, t, vof, vof
sources) in FP64 and runs the interface geometry and THINC in FP32 with FP32
intermediates (curvature, normals, forces, momentum sources, increments);
the momentum stencils, the x line solves and the Poisson solve are FP64.
Bounds, stated per result: velocity relative L2 error
<= 1e-5 against the FP64 reference after the run, max |div u| <= 1e-10 and
total-volume drift <= 1e-10.
"""
import numpy as np
import pytest

from oracle import Oracle3D
from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def interior(name, a):
    h = 2 if name == "vof" else 1
    return a[h:-h, h:-h, 1:-1]


def volume(vof, ic):
    return float(np.sum(vof * np.diff(ic.xf))) * (ic.ly / ic.ny) * (ic.lz / ic.nz)


def test_mixed_against_fp64_oracle(gpu_available):
    ic = droplets3d(32, 32, 32, ndrops=4, radii=(0.1, 0.16), seed=2)
    phys = physical_params(DROPLETS3D_ENV)
    g = Solver3D(ic, phys, precision="mixed")
    o = Oracle3D(ic, phys)
    nsteps = 20
    dts_g = g.run(nsteps)
    dts_o = o.run(nsteps)
    np.testing.assert_allclose(dts_g, dts_o, rtol=1e-5)
    errs = {k: rel_l2(interior(k, g.field(k)), interior(k, o.field(k))) for k in ("ux", "uy", "uz", "vof")}
    assert max(errs["ux"], errs["uy"], errs["uz"]) <= 1e-5, errs
    assert errs["vof"] <= 1e-5, errs
    d = g.diagnostics()
    assert d["divmax"] <= 1e-10, d
    v0 = volume(ic.vof[:, :, 1:-1], ic)
    assert abs(d["volume"] - v0) / v0 <= 1e-10, (d["volume"], v0)


def test_mixed_against_fp64_gpu(gpu_available):
    ic = droplets3d(64, 64, 64, ndrops=16, radii=(0.05, 0.1), seed=4)
    phys = physical_params(DROPLETS3D_ENV)
    m = Solver3D(ic, phys, precision="mixed")
    f = Solver3D(ic, phys)
    m.run(30)
    f.run(30)
    for k in ("ux", "uy", "uz"):
        assert rel_l2(interior(k, m.field(k)), interior(k, f.field(k))) <= 1e-5, k
    dm, df = m.diagnostics(), f.diagnostics()
    assert dm["divmax"] <= 1e-10 and df["divmax"] <= 1e-10, (dm, df)
    v0 = volume(ic.vof[:, :, 1:-1], ic)
    assert abs(dm["volume"] - v0) / v0 <= 1e-10


def test_mixed_fields_are_fp32(gpu_available):
    """FP32 intermediates download as FP64 arrays with FP32 values"""
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    g = Solver3D(ic, physical_params(DROPLETS3D_ENV), precision="mixed")
    g.integrate()
    for k in ("curv", "ifrcx", "srcuy_a"):
        a = g.field(k)
        assert np.all(np.isfinite(a)), k
        assert np.array_equal(a, a.astype(np.float32).astype(np.float64)), k
    u = g.field("ux")
    assert not np.array_equal(u, u.astype(np.float32).astype(np.float64))  # the state stays FP64
    g.set_field("curv", np.full(g.field("curv").shape, 0.1))
    assert np.allclose(g.field("curv"), np.float32(0.1))


def test_defect_corrected_poisson(gpu_available):
    """SVOF3_MIXED_DC: the Poisson solve as two FP32 passes with the FP64
    residual of the first as the right-hand side of the second.  One
    correction takes psi from FP32 accuracy to near FP64: the divergence after
    the projection stays at FP64 round-off (<= 1e-10), and the fields stay
    within the mixed path's bounds of the FP64 path"""
    ic = droplets3d(64, 64, 64, ndrops=16, radii=(0.05, 0.1), seed=4)
    phys = physical_params(DROPLETS3D_ENV)
    dc = Solver3D(ic, phys, precision="mixed_dc")
    m = Solver3D(ic, phys, precision="mixed")
    f = Solver3D(ic, phys)
    for s in (dc, m, f):
        s.run(30)
    for k in ("ux", "uy", "uz"):
        e_dc = rel_l2(interior(k, dc.field(k)), interior(k, f.field(k)))
        assert e_dc <= 1e-5, (k, e_dc)
    d = dc.diagnostics()
    assert d["divmax"] <= 1e-10, d
    v0 = volume(ic.vof[:, :, 1:-1], ic)
    assert abs(d["volume"] - v0) / v0 <= 1e-10


def test_defect_correction_reduces_the_residual(gpu_available):
    """one Poisson solve on the same predicted velocity: the corrected FP32
    pair is within 1e-9 of the FP64 solve's psi (modulo its constant), where
    one FP32 pass alone is not better than ~1e-6"""
    ic = droplets3d(32, 32, 32, ndrops=4, radii=(0.1, 0.16), seed=2)
    phys = physical_params(DROPLETS3D_ENV)
    dc = Solver3D(ic, phys, precision="mixed_dc")
    f = Solver3D(ic, phys)
    dt = f.fluid_decide_dt()
    f.interface_compute_curvature_tensor()
    f.interface_compute_force()
    f.interface_update_vof(0, dt)
    f.fluid_predict_field(0, dt)
    for k in ("ux", "uy", "uz"):
        dc.set_field(k, f.field(k))
    dc.fluid_decide_dt()
    dc.fluid_compute_potential_dft(0, dt)
    f.fluid_compute_potential_dft(0, dt)
    psi_dc, psi_f = interior("psi", dc.field("psi")), interior("psi", f.field("psi"))
    psi_dc = psi_dc - psi_dc.mean()
    psi_f = psi_f - psi_f.mean()
    e = rel_l2(psi_dc, psi_f)
    assert e <= 1e-9, e


@pytest.mark.parametrize("shape", [(32, 16, 16), (33, 8, 16), (40, 64, 32)])
def test_packed_y_transforms_match_the_fp64_solve(gpu_available, shape):
    """the mixed path's Poisson solve carries two columns per complex y
    transform (real and imaginary parts); from the same velocities its psi
    equals the FP64 path's (one real line per transform, the restatement's
    rounding) to round-off, modulo the solve's gauge constant; odd nx (a last
    block with one column) and an 8-point single-pass transform included"""
    from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params
    nx, ny, nz = shape
    ic = droplets3d(nx, ny, nz, ndrops=2, radii=(0.1, 0.15), seed=4)
    phys = physical_params(DROPLETS3D_ENV)
    out = {}
    for prec in ("fp64", "mixed"):
        s = Solver3D(ic, phys, precision=prec)
        rng = np.random.default_rng(9)
        # a velocity with divergence, so that psi is far from zero
        s.load_interior("ux", ic.ux + 0.1 * rng.standard_normal(ic.ux.shape))
        s.load_interior("uy", ic.uy + 0.1 * rng.standard_normal(ic.uy.shape))
        s.fluid_compute_potential_dft(1, 1.3e-3)
        psi = s.field("psi")[1:-1, 1:-1, :]
        out[prec] = psi - psi[:, :, 1:-1].mean()
        s.close()
    scale = np.abs(out["fp64"]).max()
    assert scale > 1e-6
    assert np.abs(out["mixed"] - out["fp64"]).max() <= 1e-12 * scale
