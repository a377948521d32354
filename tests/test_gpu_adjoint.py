"""The CUDA adjoint of the 2D step against the oracle's tangent-linear model.

Dot-product tests: for a tangent dx of a function's inputs and an adjoint
seed y_bar of its outputs, <TLM dx, y_bar> (oracle, svof_oracle_tl.inc) must
equal <dx, ADJ y_bar> (CUDA, through the C ABI) to round-off.  Both are
linearised about the same primal state: the per-function tests start the
oracle and the GPU from the same fields; the step tests drive the oracle's
tangent model along the GPU's own taped substep inputs.  The pressure's
seeds have zero sum (its additive constant is fixed by round-off).
"""
import numpy as np
import pytest

from oracle import Oracle
from simplevofsolver_b200.workloads import DROPLET2D_ENV, droplet2d, physical_params

pytestmark = pytest.mark.gpu

TOL = 1e-11


# ---- compact (adjoint) <-> storage (oracle) layouts
def cx(a, nx, ny):
    """ux faces i = 2..nx of a (ny+2, nx+1) storage array"""
    return a[1:ny + 1, 1:nx]


def cc(a, nx, ny, h=1):
    """cells of a storage array with h halo rows"""
    return a[h:h + ny, 1:nx + 1]


def fill_periodic(a, h):
    """halo rows of a (rows, cols) storage array as periodic copies"""
    ny = a.shape[0] - 2 * h
    a[:h] = a[ny:ny + h]
    a[ny + h:] = a[h:2 * h]


def setup(uniform, gravity=True, n=32):
    import torch  # noqa: F401
    from simplevofsolver_b200 import Solver
    ic = droplet2d(n, n, uniform=uniform, noise=1e-2, semi_axes=(0.25, 0.2))
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys)
    o = Oracle(ic, phys)
    if gravity:
        g.set_gravity(-0.9, 0.15)
        o.set_gravity(-0.9, 0.15)
    g.adjoint_reset()
    g.synchronize()
    return g, o, o.tangent()


def put(g, name, x):
    import torch
    v = g.adjoint_view(name)
    v.copy_(torch.as_tensor(np.ascontiguousarray(x), device="cuda"))
    torch.cuda.synchronize()


def get(g, name):
    import torch
    g.synchronize()
    torch.cuda.synchronize()
    return g.adjoint_view(name).cpu().numpy().copy()


def rnd(rng, shape):
    return rng.standard_normal(shape)


def zero_mean(x):
    return x - x.mean()


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def tangent_cells(tan, name, x, h):
    a = tan.field(name)
    a[...] = 0.
    cc(a, tan.nx, tan.ny, h)[...] = x


@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("rk", [0, 2])
def test_update_pressure_and_correct_velocity(gpu_available, uniform, rk):
    g, o, tan = setup(uniform)
    nx, ny, dt = g.nx, g.ny, 1.3e-3
    rng = np.random.default_rng(1)
    dp, dpsi = rnd(rng, (ny, nx)), rnd(rng, (ny, nx))
    dux, duy = rnd(rng, (ny, nx - 1)), rnd(rng, (ny, nx))
    pb, uxb, uyb = zero_mean(rnd(rng, (ny, nx))), rnd(rng, (ny, nx - 1)), rnd(rng, (ny, nx))
    # tangent: psi with its Neumann ghosts and periodic halo, then the two linear functions
    psi = tan.field("psi")
    psi[...] = 0.
    cc(psi, nx, ny)[...] = dpsi
    psi[:, 0] = psi[:, 1]
    psi[:, nx + 1] = psi[:, nx]
    fill_periodic(psi, 1)
    cx(tan.field("ux"), nx, ny)[...] = dux
    cc(tan.field("uy"), nx, ny)[...] = duy
    cc(tan.field("p"), nx, ny)[...] = dp
    tan.init_boundaries()
    tan.correct(rk, dt)
    tan.update_pressure(rk, dt)
    lhs = (np.sum(cx(tan.field("ux"), nx, ny) * uxb) + np.sum(cc(tan.field("uy"), nx, ny) * uyb)
           + np.sum(cc(tan.field("p"), nx, ny) * pb))
    put(g, "ux", uxb)
    put(g, "uy", uyb)
    put(g, "p", pb)
    g.adjoint_fluid_update_pressure(rk, dt)
    g.adjoint_fluid_correct_velocity(rk, dt)
    rhs = (np.sum(dux * get(g, "ux")) + np.sum(duy * get(g, "uy")) + np.sum(dp * get(g, "p"))
           + np.sum(dpsi * get(g, "psi")))
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


@pytest.mark.parametrize("uniform", [True, False])
def test_compute_potential(gpu_available, uniform):
    g, o, tan = setup(uniform)
    nx, ny, dt, rk = g.nx, g.ny, 1.1e-3, 1
    rng = np.random.default_rng(2)
    dux, duy = rnd(rng, (ny, nx - 1)), rnd(rng, (ny, nx))
    psib = zero_mean(rnd(rng, (ny, nx)))
    cx(tan.field("ux"), nx, ny)[...] = dux
    cc(tan.field("uy"), nx, ny)[...] = duy
    tan.init_boundaries()
    tan.potential(rk, dt)
    lhs = np.sum(cc(tan.field("psi"), nx, ny) * psib)
    put(g, "psi", psib)
    g.adjoint_fluid_compute_potential(rk, dt)
    rhs = np.sum(dux * get(g, "ux")) + np.sum(duy * get(g, "uy"))
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)
    assert np.all(get(g, "psi") == 0.)


@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("rk", [0, 2])
def test_predict_field(gpu_available, uniform, rk):
    g, o, tan = setup(uniform)
    nx, ny, dt = g.nx, g.ny, 1.2e-3
    rng = np.random.default_rng(3)
    d = {"ux": rnd(rng, (ny, nx - 1)), "uy": rnd(rng, (ny, nx)), "p": rnd(rng, (ny, nx)),
         "vof": rnd(rng, (ny, nx)), "ifrcx": rnd(rng, (ny, nx - 1)), "ifrcy": rnd(rng, (ny, nx)),
         "sbx": rnd(rng, (ny, nx - 1)), "sby": rnd(rng, (ny, nx))}
    b = {"ux": rnd(rng, (ny, nx - 1)), "uy": rnd(rng, (ny, nx)), "sax": rnd(rng, (ny, nx - 1)),
         "say": rnd(rng, (ny, nx))}
    cx(tan.field("ux"), nx, ny)[...] = d["ux"]
    cc(tan.field("uy"), nx, ny)[...] = d["uy"]
    cc(tan.field("p"), nx, ny)[...] = d["p"]
    cc(tan.field("vof"), nx, ny, 2)[...] = d["vof"]
    tan.init_boundaries()
    tan.field("ifrcx")[...] = d["ifrcx"]
    tan.field("ifrcy")[...] = d["ifrcy"]
    # src_b of this substep is the current src_a (moved by reset_srcs)
    tan.field("srcux0")[...] = d["sbx"]
    tan.field("srcuy0")[...] = d["sby"]
    dgrav = 0.23    # tangent of the vof buoyancy coefficient
    tan.predict(rk, dt, dgrav)
    lhs = (np.sum(cx(tan.field("ux"), nx, ny) * b["ux"]) + np.sum(cc(tan.field("uy"), nx, ny) * b["uy"])
           + np.sum(tan.field("srcux0") * b["sax"]) + np.sum(tan.field("srcuy0") * b["say"]))
    put(g, "ux", b["ux"])
    put(g, "uy", b["uy"])
    put(g, "srcux_a", b["sax"])
    put(g, "srcuy_a", b["say"])
    g.adjoint_fluid_predict_field(rk, dt)
    rhs = (np.sum(d["ux"] * get(g, "ux")) + np.sum(d["uy"] * get(g, "uy")) + np.sum(d["p"] * get(g, "p"))
           + np.sum(d["vof"] * get(g, "vof")) + np.sum(d["ifrcx"] * get(g, "ifrcx"))
           + np.sum(d["ifrcy"] * get(g, "ifrcy")) + dgrav * g.adjoint_gravity())
    if rk != 0:
        rhs += np.sum(d["sbx"] * get(g, "srcux_a")) + np.sum(d["sby"] * get(g, "srcuy_a"))
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def interfacial_mask(o, nx, ny):
    v = cc(o.field("vof"), nx, ny, 2)
    return (v >= 1e-8) & (v <= 1 - 1e-8)


@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("rk", [0, 1])
def test_update_vof(gpu_available, uniform, rk):
    g, o, tan = setup(uniform)
    nx, ny, dt = g.nx, g.ny, 1.0e-3
    g.interface_compute_curvature_tensor()
    o.curvature_tensor()
    rng = np.random.default_rng(4)
    inter = interfacial_mask(o, nx, ny)
    dn = rnd(rng, (ny, nx, 3)) * inter[..., None]
    d = {"ux": rnd(rng, (ny, nx - 1)), "uy": rnd(rng, (ny, nx)), "vof": rnd(rng, (ny, nx)) * 1e-3,
         "sb": rnd(rng, (ny, nx))}
    b = {"vof": rnd(rng, (ny, nx)), "sa": rnd(rng, (ny, nx))}
    cx(tan.field("ux"), nx, ny)[...] = d["ux"]
    cc(tan.field("uy"), nx, ny)[...] = d["uy"]
    cc(tan.field("vof"), nx, ny, 2)[...] = d["vof"]
    tan.init_boundaries()
    nrm = tan.field("normal")
    nrm[1:ny + 1] = dn
    nrm[0] = nrm[ny]
    nrm[ny + 1] = nrm[1]
    tan.field("src0")[...] = d["sb"]
    tan.update_vof(rk, dt)
    lhs = np.sum(cc(tan.field("vof"), nx, ny, 2) * b["vof"]) + np.sum(tan.field("src0") * b["sa"])
    put(g, "vof", b["vof"])
    put(g, "src_a", b["sa"])
    g.adjoint_interface_update_vof(rk, dt)
    rhs = (np.sum(d["ux"] * get(g, "ux")) + np.sum(d["uy"] * get(g, "uy")) + np.sum(d["vof"] * get(g, "vof"))
           + np.sum(dn * get(g, "normal")))
    if rk != 0:
        rhs += np.sum(d["sb"] * get(g, "src_a"))
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


@pytest.mark.parametrize("uniform", [True, False])
def test_force(gpu_available, uniform):
    g, o, tan = setup(uniform)
    nx, ny = g.nx, g.ny
    g.interface_compute_curvature_tensor()
    o.curvature_tensor()
    rng = np.random.default_rng(5)
    dvof, dcurv, dten = rnd(rng, (ny, nx)), rnd(rng, (ny, nx)), 0.37
    bx, by = rnd(rng, (ny, nx - 1)), rnd(rng, (ny, nx))
    cc(tan.field("vof"), nx, ny, 2)[...] = dvof
    tan.init_boundaries()
    cu = tan.field("curv")
    cu[...] = 0.
    cc(cu, nx, ny)[...] = dcurv
    fill_periodic(cu, 1)
    tan.force(dten)
    lhs = np.sum(tan.field("ifrcx") * bx) + np.sum(tan.field("ifrcy") * by)
    put(g, "ifrcx", bx)
    put(g, "ifrcy", by)
    g.adjoint_interface_compute_force()
    rhs = np.sum(dvof * get(g, "vof")) + np.sum(dcurv * get(g, "curv")) + dten * g.adjoint_tension()
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


@pytest.mark.parametrize("uniform", [True, False])
def test_curvature_tensor(gpu_available, uniform):
    g, o, tan = setup(uniform)
    nx, ny = g.nx, g.ny
    g.interface_compute_curvature_tensor()
    o.curvature_tensor()
    rng = np.random.default_rng(6)
    inter = interfacial_mask(o, nx, ny)
    dvof = rnd(rng, (ny, nx))
    nb = rnd(rng, (ny, nx, 3)) * inter[..., None]
    kb = rnd(rng, (ny, nx))
    cc(tan.field("vof"), nx, ny, 2)[...] = dvof
    tan.init_boundaries()
    tan.curvature_tensor()
    lhs = np.sum(tan.field("normal")[1:ny + 1] * nb) + np.sum(cc(tan.field("curv"), nx, ny) * kb)
    put(g, "normal", nb)
    put(g, "curv", kb)
    g.adjoint_interface_compute_curvature_tensor()
    rhs = np.sum(dvof * get(g, "vof"))
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def tangent_step_along(o, tan, tape, rk_fields, dt, dten, dgrav=0.0):
    """one step of the oracle's tangent model linearised about the GPU's taped
    substep inputs (ux, uy, vof of each substep; the predictor's vof is the
    one after the substep's advection: the next entry's)"""
    for rk in range(3):
        for k in ("ux", "uy", "vof"):
            o.field(k)[...] = rk_fields[rk][k]
        o.curvature_tensor()
        tan.curvature_tensor()
        tan.force(dten)
        tan.update_vof(rk, dt)
        o.field("vof")[...] = rk_fields[rk + 1]["vof"]
        tan.predict(rk, dt, dgrav)
        tan.potential(rk, dt)
        tan.correct(rk, dt)
        tan.update_pressure(rk, dt)


def taped_fields(g, tape):
    """split one step's tape into the substep inputs (storage layouts) and,
    as a fourth entry, the step's final vof"""
    from simplevofsolver_b200 import storage_shape
    nx, ny = g.nx, g.ny
    t = tape.cpu().numpy()
    sizes = [np.prod(storage_shape(k, nx, ny)) for k in ("ux", "uy", "vof")]
    st = sum(sizes)
    assert t.size == 3 * st + sizes[2]
    out = []
    for rk in range(3):
        base = rk * st
        d = {}
        for k, n in zip(("ux", "uy", "vof"), sizes):
            d[k] = t[base:base + n].reshape(storage_shape(k, nx, ny))
            base += n
        out.append(d)
    out.append({"vof": t[3 * st:].reshape(storage_shape("vof", nx, ny))})
    return out


@pytest.mark.parametrize("uniform,gravity,steps", [(True, False, 1), (False, True, 1), (False, True, 3)])
def test_step_dot_product(gpu_available, uniform, gravity, steps):
    import torch
    g, o, tan = setup(uniform, gravity)
    nx, ny = g.nx, g.ny
    dt = g.fluid_decide_dt()
    tapes = [torch.empty(g.tape_count(), dtype=torch.float64, device="cuda") for _ in range(steps)]
    torch.cuda.synchronize()
    for k in range(steps):
        g.integrate_fixed(dt, tapes[k].data_ptr())
    g.synchronize()
    rng = np.random.default_rng(7)
    d0 = {"ux": rnd(rng, (ny, nx - 1)), "uy": rnd(rng, (ny, nx)), "p": rnd(rng, (ny, nx)),
          "vof": rnd(rng, (ny, nx)) * interfacial_mask(o, nx, ny)}
    dten, dgrav = 0.21, -0.17
    b = {"ux": rnd(rng, (ny, nx - 1)), "uy": rnd(rng, (ny, nx)), "p": zero_mean(rnd(rng, (ny, nx))),
         "vof": rnd(rng, (ny, nx))}
    # tangent model along the GPU trajectory
    cx(tan.field("ux"), nx, ny)[...] = d0["ux"]
    cc(tan.field("uy"), nx, ny)[...] = d0["uy"]
    cc(tan.field("p"), nx, ny)[...] = d0["p"]
    cc(tan.field("vof"), nx, ny, 2)[...] = d0["vof"]
    tan.init_boundaries()
    for k in range(steps):
        tangent_step_along(o, tan, tapes[k], taped_fields(g, tapes[k]), dt, dten, dgrav)
    lhs = (np.sum(cx(tan.field("ux"), nx, ny) * b["ux"]) + np.sum(cc(tan.field("uy"), nx, ny) * b["uy"])
           + np.sum(cc(tan.field("p"), nx, ny) * b["p"]) + np.sum(cc(tan.field("vof"), nx, ny, 2) * b["vof"]))
    # adjoint
    for k in ("ux", "uy", "p", "vof"):
        put(g, k, b[k])
    for k in reversed(range(steps)):
        g.adjoint_step(tapes[k].data_ptr(), dt)
    rhs = (sum(np.sum(d0[k] * get(g, k)) for k in ("ux", "uy", "p", "vof")) + dten * g.adjoint_tension()
           + dgrav * g.adjoint_gravity())
    assert rel(lhs, rhs) <= 1e-10, (lhs, rhs)
    g.close()
