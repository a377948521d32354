"""The CUDA adjoint of the 3D step (FP64 path) against central differences of
the CUDA forward.

The 3D path has no tangent model in the oracle; its forward is pinned to the
3D restatement function by function (test_gpu3d_parity.py), so each
transpose is checked against the forward it transposes: for inputs x, a
tangent d and an adjoint seed y_bar, <y_bar, (F(x + e d) - F(x - e d)) / 2e>
(the GPU forward through the C ABI) must equal <d, F^T y_bar> (the GPU
adjoint).  The linear functions (projection, pressure update, Poisson solve)
and the quadratic ones (momentum right-hand sides and x solves, CSF force)
have exact central differences, so those tests take e = 1 and round-off
tolerances; the THINC fluxes and the geometry are smooth but not
polynomial and take a small e, with the vof tangent confined to interfacial
cells away from the 1e-8 thresholds (the branch sets do not change).  The
step test differentiates two full steps with respect to a discretely
divergence-free initial velocity direction and the surface-tension
coefficient.
"""
import numpy as np
import pytest

from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params

pytestmark = pytest.mark.gpu

TOL_LINEAR = 1e-10


def make(seed=3):
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=seed)
    phys = physical_params(DROPLETS3D_ENV)
    g = Solver3D(ic, phys)
    return ic, phys, g


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


# ---- layouts: compact (adjoint) <-> restart interior (load_interior) and storage
def embed(name, c, nx):
    """compact (nz, ny, nx-1 | nx) -> restart interior with zero x ghosts"""
    nz, ny = c.shape[:2]
    out = np.zeros((nz, ny, nx + 1 if name == "ux" else nx + 2))
    if name == "ux":
        out[..., 1:nx] = c
    else:
        out[..., 1:nx + 1] = c
    return out


def compact(name, a, nx):
    return a[..., 1:nx] if name == "ux" else a[..., 1:nx + 1]


def fill_periodic(a):
    """the one-deep y and z halos of a storage array (axes 0 = z, 1 = y)"""
    nz, ny = a.shape[0] - 2, a.shape[1] - 2
    a[:, 0] = a[:, ny]
    a[:, ny + 1] = a[:, 1]
    a[0] = a[nz]
    a[nz + 1] = a[1]


def set_storage_interior(g, name, c):
    """writes the interior of a halo'd storage field (curv: (nz, ny, nx);
    normal: (nz, ny, nx, 4)) with periodic halo copies"""
    s = g.field(name)
    if name == "normal":
        s[1:-1, 1:-1] = c
    else:
        s[1:-1, 1:-1, 1:g.nx + 1] = c
    fill_periodic(s)
    g.set_field(name, s)


def storage_interior(g, name):
    s = g.field(name)
    return s[1:-1, 1:-1].copy() if name == "normal" else s[1:-1, 1:-1, 1:g.nx + 1].copy()


def put_adj(g, name, x):
    import torch
    g.synchronize()
    g.adjoint_view(name).copy_(torch.as_tensor(np.ascontiguousarray(x), device="cuda"))
    torch.cuda.synchronize()


def get_adj(g, name):
    import torch
    g.synchronize()
    torch.cuda.synchronize()
    return g.adjoint_view(name).cpu().numpy().copy()


def shapes(g):
    nx, ny, nz = g.nx, g.ny, g.nz
    return (nz, ny, nx - 1), (nz, ny, nx)


class State:
    """a base state (restart interiors, storage interiors, compact arrays)
    and its loading with a tangent scaled by e"""

    INTERIOR = ("ux", "uy", "uz", "p", "psi", "vof", "t")
    STORAGE = ("curv", "normal")

    def __init__(self, g, names):
        self.g = g
        self.base = {}
        for n in names:
            if n in self.INTERIOR:
                self.base[n] = g.interior(n)
            elif n in self.STORAGE:
                self.base[n] = storage_interior(g, n)
            else:
                self.base[n] = g.field(n)

    def load(self, d=None, e=0.0):
        g = self.g
        for n, b in self.base.items():
            x = b.copy()
            if d is not None and n in d:
                x = x + e * (embed(n, d[n], g.nx) if n in self.INTERIOR else d[n])
            if n in self.INTERIOR:
                g.load_interior(n, x)
            elif n in self.STORAGE:
                set_storage_interior(g, n, x)
            else:
                g.set_field(n, x)
        g.synchronize()


def read(g, n):
    return compact(n, g.interior(n), g.nx) if n in State.INTERIOR else (
        storage_interior(g, n) if n in State.STORAGE else g.field(n))


def central(state, d, e, run, outs, seeds):
    """<seeds, (F(x + e d) - F(x - e d)) / 2e> over the outputs outs"""
    vals = []
    for sgn in (+1.0, -1.0):
        state.load(d, sgn * e)
        run()
        vals.append({n: read(state.g, n) for n in outs})
    return sum(float(np.sum(seeds[n] * (vals[0][n] - vals[1][n]) / (2.0 * e))) for n in outs)


def interfacial_cells(g, lo=1e-4):
    v = compact("vof", g.interior("vof"), g.nx)
    return (v > lo) & (v < 1.0 - lo)


@pytest.mark.parametrize("rk", [0, 2])
def test_update_pressure_and_correct_velocity(gpu_available, rk):
    ic, phys, g = make()
    dt = 1.3e-3
    rng = np.random.default_rng(1)
    fs, cs = shapes(g)
    d = {"ux": rng.standard_normal(fs), "uy": rng.standard_normal(cs), "uz": rng.standard_normal(cs),
         "p": rng.standard_normal(cs), "psi": rng.standard_normal(cs)}
    g.load_interior("psi", embed("psi", rng.standard_normal(cs), g.nx))
    st = State(g, ("ux", "uy", "uz", "p", "psi"))
    seeds = {"ux": rng.standard_normal(fs), "uy": rng.standard_normal(cs), "uz": rng.standard_normal(cs),
             "p": rng.standard_normal(cs)}

    def run():
        g.fluid_correct_velocity(rk, dt)
        g.fluid_update_pressure(rk, dt)

    lhs = central(st, d, 1.0, run, ("ux", "uy", "uz", "p"), seeds)
    st.load()
    g.adjoint_reset()
    for n, v in seeds.items():
        put_adj(g, n, v)
    g.adjoint_fluid_update_pressure(rk, dt)
    g.adjoint_fluid_correct_velocity(rk, dt)
    rhs = sum(float(np.sum(d[n] * get_adj(g, n))) for n in ("ux", "uy", "uz", "p", "psi"))
    assert rel(lhs, rhs) <= TOL_LINEAR, (lhs, rhs)


@pytest.mark.parametrize("rk", [0, 1])
def test_compute_potential(gpu_available, rk):
    ic, phys, g = make()
    dt = 1.1e-3
    rng = np.random.default_rng(2)
    fs, cs = shapes(g)
    d = {"ux": rng.standard_normal(fs), "uy": rng.standard_normal(cs), "uz": rng.standard_normal(cs)}
    st = State(g, ("ux", "uy", "uz"))
    psib = rng.standard_normal(cs)
    psib -= psib.mean()
    vals = []
    for sgn in (+1.0, -1.0):
        st.load(d, sgn)
        g.fluid_compute_potential_dft(rk, dt)
        vals.append(read(g, "psi"))
    dpsi = (vals[0] - vals[1]) / 2.0
    # psi is fixed up to a constant (the singular mode's round-off)
    lhs = float(np.sum(psib * (dpsi - dpsi.mean())))
    st.load()
    g.adjoint_reset()
    put_adj(g, "psi", psib)
    g.adjoint_fluid_compute_potential_dft(rk, dt)
    rhs = sum(float(np.sum(d[n] * get_adj(g, n))) for n in ("ux", "uy", "uz"))
    assert rel(lhs, rhs) <= TOL_LINEAR, (lhs, rhs)
    assert np.all(get_adj(g, "psi") == 0.0)


@pytest.mark.parametrize("rk", [0, 2])
def test_predict_field(gpu_available, rk):
    """with the vof buoyancy extension on: the source is bilinear in (vof,
    grav), so the vof and grav directions are differenced separately"""
    ic, phys, g = make()
    dt = 1.2e-3
    rng = np.random.default_rng(3)
    fs, cs = shapes(g)
    grav, dgrav = -0.9, 0.31
    g.set_gravity(grav, 0.2)
    # src_b of this substep is the current src_a (the call swaps them first)
    for n, sh in (("srcux_a", fs), ("srcuy_a", cs), ("srcuz_a", cs)):
        g.set_field(n, rng.standard_normal(sh))
    for n, sh in (("ifrcx", fs), ("ifrcy", cs), ("ifrcz", cs)):
        g.set_field(n, rng.standard_normal(sh))
    names = ("ux", "uy", "uz", "p", "vof", "ifrcx", "ifrcy", "ifrcz", "srcux_a", "srcuy_a", "srcuz_a")
    st = State(g, names)
    d = {n: rng.standard_normal(st.base[n].shape if n not in State.INTERIOR else
                                (fs if n == "ux" else cs)) for n in names}
    seeds = {n: rng.standard_normal(fs if n in ("ux", "srcux_a") else cs)
             for n in ("ux", "uy", "uz", "srcux_a", "srcuy_a", "srcuz_a")}

    def run():
        g.fluid_predict_field(rk, dt)

    lhs = central(st, d, 1.0, run, tuple(seeds), seeds)
    vals = []
    for sgn in (+1.0, -1.0):
        st.load()
        g.set_gravity(grav + sgn * dgrav, 0.2)
        run()
        vals.append({n: read(g, n) for n in seeds})
    lhs_g = sum(float(np.sum(seeds[n] * (vals[0][n] - vals[1][n]) / 2.0)) for n in seeds)
    g.set_gravity(grav, 0.2)
    st.load()
    g.adjoint_reset()
    for n, v in seeds.items():
        put_adj(g, n, v)
    g.adjoint_fluid_predict_field(rk, dt)
    rhs_g = dgrav * g.adjoint_gravity()
    assert rel(lhs_g, rhs_g) <= 1e-9, ("gravity", lhs_g, rhs_g)
    rhs = 0.0
    for n in ("ux", "uy", "uz", "p", "vof", "ifrcx", "ifrcy", "ifrcz"):
        rhs += float(np.sum(d[n] * get_adj(g, n)))
    if rk != 0:
        for n in ("srcux_a", "srcuy_a", "srcuz_a"):
            rhs += float(np.sum(d[n] * get_adj(g, n)))
    assert rel(lhs, rhs) <= 1e-9, (lhs, rhs)


@pytest.mark.parametrize("rk", [0, 1])
def test_update_vof(gpu_available, rk):
    ic, phys, g = make()
    dt = 1.0e-3
    rng = np.random.default_rng(4)
    fs, cs = shapes(g)
    g.interface_compute_curvature_tensor()
    g.set_field("src_a", rng.standard_normal(cs))
    mask = interfacial_cells(g)
    assert mask.sum() > 50
    names = ("ux", "uy", "uz", "vof", "normal", "src_a")
    st = State(g, names)
    d = {"ux": rng.standard_normal(fs), "uy": rng.standard_normal(cs), "uz": rng.standard_normal(cs),
         "vof": rng.standard_normal(cs) * mask, "normal": rng.standard_normal(cs + (4,)) * mask[..., None],
         "src_a": rng.standard_normal(cs)}
    seeds = {"vof": rng.standard_normal(cs), "src_a": rng.standard_normal(cs)}

    def run():
        g.interface_update_vof(rk, dt)

    lhs = central(st, d, 1e-6, run, ("vof", "src_a"), seeds)
    st.load()
    g.adjoint_reset()
    put_adj(g, "vof", seeds["vof"])
    put_adj(g, "src_a", seeds["src_a"])
    g.adjoint_interface_update_vof(rk, dt)
    rhs = sum(float(np.sum(d[n] * get_adj(g, n))) for n in ("ux", "uy", "uz", "vof", "normal"))
    if rk != 0:
        rhs += float(np.sum(d["src_a"] * get_adj(g, "src_a")))
    assert rel(lhs, rhs) <= 1e-7, (lhs, rhs)


def test_compute_force(gpu_available):
    ic, phys, g = make()
    rng = np.random.default_rng(5)
    fs, cs = shapes(g)
    g.interface_compute_curvature_tensor()
    st = State(g, ("vof", "curv"))
    d = {"vof": rng.standard_normal(cs), "curv": rng.standard_normal(cs)}
    dten = 0.37
    seeds = {"ifrcx": rng.standard_normal(fs), "ifrcy": rng.standard_normal(cs), "ifrcz": rng.standard_normal(cs)}
    ten = phys["tension"]
    # the force is trilinear in (tension, vof, curv): central differences
    # are exact along (vof, curv) at fixed tension and along the tension alone
    lhs = 0.0
    for dd, dt_ in ((d, 0.0), (None, dten)):
        vals = []
        for sgn in (+1.0, -1.0):
            st.load(dd, sgn)
            g.set_tension(ten + sgn * dt_)
            g.interface_compute_force()
            vals.append({n: g.field(n) for n in seeds})
        lhs += sum(float(np.sum(seeds[n] * (vals[0][n] - vals[1][n]) / 2.0)) for n in seeds)
    g.set_tension(ten)
    st.load()
    g.adjoint_reset()
    for n, v in seeds.items():
        put_adj(g, n, v)
    g.adjoint_interface_compute_force()
    rhs = (float(np.sum(d["vof"] * get_adj(g, "vof"))) + float(np.sum(d["curv"] * get_adj(g, "curv")))
           + dten * g.adjoint_tension())
    assert rel(lhs, rhs) <= TOL_LINEAR, (lhs, rhs)


def test_compute_curvature_tensor(gpu_available):
    ic, phys, g = make()
    rng = np.random.default_rng(6)
    fs, cs = shapes(g)
    mask = interfacial_cells(g)
    inter = interfacial_cells(g, 1e-8)
    st = State(g, ("vof",))
    d = {"vof": rng.standard_normal(cs) * mask}
    seeds = {"normal": rng.standard_normal(cs + (4,)) * inter[..., None], "curv": rng.standard_normal(cs)}

    def run():
        g.interface_compute_curvature_tensor()

    lhs = central(st, d, 1e-7, run, ("normal", "curv"), seeds)
    st.load()
    g.interface_compute_curvature_tensor()
    g.adjoint_reset()
    put_adj(g, "normal", seeds["normal"])
    put_adj(g, "curv", seeds["curv"])
    g.adjoint_interface_compute_curvature_tensor()
    rhs = float(np.sum(d["vof"] * get_adj(g, "vof")))
    assert rel(lhs, rhs) <= 1e-6, (lhs, rhs)


@pytest.mark.parametrize("direction", ["velocity", "tension", "gravity"])
def test_two_steps(gpu_available, direction):
    """two full steps (fixed dt), the vof buoyancy extension on: the
    directional derivative along a divergence-free velocity, the tension and
    the buoyancy coefficient, each against the adjoint"""
    import torch
    ic, phys, g = make()
    nx = g.nx
    fs, cs = shapes(g)
    dt = g.fluid_decide_dt()
    rng = np.random.default_rng(7)
    # a discretely divergence-free direction: the generator's velocity of another seed
    dirn = droplets3d(32, 16, 16, ndrops=1, radii=(0.12, 0.13), seed=11)
    d = {"ux": compact("ux", dirn.ux, nx), "uy": compact("uy", dirn.uy, nx), "uz": compact("uz", dirn.uz, nx)}
    if direction != "velocity":
        d = {k: 0.0 * v for k, v in d.items()}
    dten = 0.3 * phys["tension"] if direction == "tension" else 0.0
    grav, dgrav = -0.9, (0.2 if direction == "gravity" else 0.0)
    seeds = {"ux": rng.standard_normal(fs), "uy": rng.standard_normal(cs), "uz": rng.standard_normal(cs),
             "p": rng.standard_normal(cs)}
    seeds["p"] -= seeds["p"].mean()
    yc = (np.arange(g.ny) + 0.5) / g.ny
    seeds["vof"] = np.broadcast_to(yc[None, :, None], cs).copy()
    nsteps = 2

    def J(e):
        for n, v in ic.fields().items():
            x = v.copy()
            if n in d:
                x = x + e * embed(n, d[n], nx)
            g.load_interior(n, x)
        g.set_tension(phys["tension"] + e * dten)
        g.set_gravity(grav + e * dgrav, 0.15)
        for _ in range(nsteps):
            g.integrate_fixed(dt)
        g.synchronize()
        return sum(float(np.sum(seeds[n] * read(g, n))) for n in seeds)

    e = 1e-6
    lhs = (J(e) - J(-e)) / (2 * e)
    # the adjoint: recorded forward, then the step adjoints in reverse
    for n, v in ic.fields().items():
        g.load_interior(n, v)
    g.set_tension(phys["tension"])
    g.set_gravity(grav, 0.15)
    tapes = [torch.empty(g.tape_count(), dtype=torch.float64, device="cuda") for _ in range(nsteps)]
    for t in tapes:
        g.integrate_fixed(dt, t.data_ptr())
    g.synchronize()
    g.adjoint_reset()
    for n, v in seeds.items():
        put_adj(g, n, v)
    for t in reversed(tapes):
        g.adjoint_step(t.data_ptr(), dt)
    rhs = (sum(float(np.sum(d[n] * get_adj(g, n))) for n in d) + dten * g.adjoint_tension()
           + dgrav * g.adjoint_gravity())
    assert rel(lhs, rhs) <= 1e-5, (lhs, rhs)


def test_mixed_path_transposes_use_fp64_geometry(gpu_available):
    """on the mixed path the adjoint computes in FP64 about FP64 geometry
    recomputed from vof: the force transpose of the same state and seeds is
    the FP64 path's, bit for bit"""
    from simplevofsolver_b200 import physical_params
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    rng = np.random.default_rng(8)
    seeds = {"ifrcx": rng.standard_normal((16, 16, 31)), "ifrcy": rng.standard_normal((16, 16, 32)),
             "ifrcz": rng.standard_normal((16, 16, 32))}
    out = []
    for prec in ("fp64", "mixed"):
        g = Solver3D(ic, physical_params(DROPLETS3D_ENV), precision=prec)
        g.interface_compute_curvature_tensor()
        g.adjoint_reset()
        for n, v in seeds.items():
            put_adj(g, n, v)
        g.adjoint_interface_compute_force()
        out.append((get_adj(g, "vof"), get_adj(g, "curv"), g.adjoint_tension()))
    for a_, b_ in zip(out[0], out[1]):
        assert np.array_equal(a_, b_)


def test_rollout3d_gradient_and_checkpoints(gpu_available):
    """torch autograd through Rollout3D (6 steps, checkpoints every 4: a
    partial last segment): the gradient along a divergence-free velocity
    direction and the tension against central differences; K = 1 and 6 give
    the same gradients as K = 4 (the recompute is deterministic)"""
    import torch
    from simplevofsolver_b200.adjoint import Rollout3D, rollout3d
    ic, phys, g = make()
    nx = g.nx
    dts = [g.fluid_decide_dt()] * 6
    dev = dict(dtype=torch.float64, device="cuda")
    x0 = {n: torch.tensor(compact(n, getattr(ic, n), nx), **dev) for n in ("ux", "uy", "uz", "vof")}
    x0["ten"] = torch.tensor(phys["tension"], **dev)
    yc = torch.tensor((np.arange(g.ny) + 0.5) / g.ny, **dev)

    def objective(out):
        ux, uy, uz, vof, p = out
        return (torch.sum(vof * yc[None, :, None]) + 0.1 * (torch.sum(ux * ux) + torch.sum(uy * uy)
                                                            + torch.sum(uz * uz)))

    def grads(K):
        for n, v in ic.fields().items():     # the rollout takes p and t from the solver
            g.load_interior(n, v)
        r = Rollout3D(g, dts, K)
        xs = {k: v.clone().requires_grad_(k != "vof") for k, v in x0.items()}
        J = objective(rollout3d(xs["ux"], xs["uy"], xs["uz"], xs["vof"], xs["ten"], r))
        J.backward()
        return r, {k: xs[k].grad.clone() for k in ("ux", "uy", "uz", "ten")}

    r, gr = grads(4)
    dirn = droplets3d(32, 16, 16, ndrops=1, radii=(0.12, 0.13), seed=11)
    d = {n: torch.tensor(compact(n, getattr(dirn, n), nx), **dev) for n in ("ux", "uy", "uz")}
    dten = 0.3 * phys["tension"]

    def J(e):
        with torch.no_grad():
            out = r.forward(x0["ux"] + e * d["ux"], x0["uy"] + e * d["uy"], x0["uz"] + e * d["uz"], x0["vof"],
                            float(x0["ten"]) + e * dten, keep_checkpoints=False)
            return float(objective(out))

    e = 1e-6
    fd = (J(e) - J(-e)) / (2 * e)
    ad = sum(float(torch.sum(gr[n] * d[n])) for n in d) + dten * float(gr["ten"])
    assert rel(fd, ad) <= 1e-5, (fd, ad)
    for K in (1, 6):
        _, gk = grads(K)
        for n in gr:
            assert torch.equal(gk[n], gr[n]), (K, n)


def test_defect_corrected_path_adjoint(gpu_available):
    """the adjoint on the defect-corrected precision (its forward's Poisson
    passes FP32; the adjoint's second solve FP64): two taped steps, the
    directional derivative along a divergence-free velocity equals the mixed
    path's within their trajectories' difference; a negative gradient floor
    is refused"""
    import torch
    from simplevofsolver_b200 import SvofError, physical_params
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    dirn = droplets3d(32, 16, 16, ndrops=1, radii=(0.12, 0.13), seed=11)
    d = {n: compact(n, getattr(dirn, n), 32) for n in ("ux", "uy", "uz")}
    dd = {}
    for prec in ("mixed", "mixed_dc"):
        g = Solver3D(ic, phys, precision=prec)
        dt = 1.0e-3
        tapes = [torch.empty(g.tape_count(), dtype=torch.float64, device="cuda") for _ in range(2)]
        for t in tapes:
            g.integrate_fixed(dt, t.data_ptr())
        g.synchronize()
        g.adjoint_reset()
        rng = np.random.default_rng(12)
        put_adj(g, "ux", rng.standard_normal((16, 16, 31)))
        put_adj(g, "uy", rng.standard_normal((16, 16, 32)))
        for t in reversed(tapes):
            g.adjoint_step(t.data_ptr(), dt)
        dd[prec] = sum(float(np.sum(d[n] * get_adj(g, n))) for n in d)
        with pytest.raises(SvofError, match="non-negative"):
            g.adjoint_set_gradient_floor(-1.0)
        g.close()
    assert np.isfinite(dd["mixed_dc"])
    assert rel(dd["mixed"], dd["mixed_dc"]) <= 1e-4, dd


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_fp32_intermediates(gpu_available, prec):
    """the adjoint with FP32 intermediates (svof3d_adjoint_set_precision) against
    the FP64 intermediates with the same gradient floor: two taped steps, the
    directional derivatives along a divergence-free velocity, the tension
    and the buoyancy coefficient agree to FP32 round-off; the FP32
    intermediates are not exposed as FP64 views"""
    import torch
    from simplevofsolver_b200 import SvofError, physical_params
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    dirn = droplets3d(32, 16, 16, ndrops=1, radii=(0.12, 0.13), seed=11)
    d = {n: compact(n, getattr(dirn, n), 32) for n in ("ux", "uy", "uz")}
    out = {}
    for adj in ("fp64", "fp32"):
        g = Solver3D(ic, phys, precision=prec)
        g.set_gravity(-0.9, 0.15)
        g.adjoint_set_precision(adj)
        g.adjoint_set_gradient_floor(1e-5)
        dt = 1.0e-3
        tapes = [torch.empty(g.tape_count(), dtype=torch.float64, device="cuda") for _ in range(2)]
        for t in tapes:
            g.integrate_fixed(dt, t.data_ptr())
        g.synchronize()
        g.adjoint_reset()
        rng = np.random.default_rng(13)
        put_adj(g, "ux", rng.standard_normal((16, 16, 31)))
        put_adj(g, "uy", rng.standard_normal((16, 16, 32)))
        put_adj(g, "vof", np.broadcast_to(((np.arange(16) + 0.5) / 16)[None, :, None], (16, 16, 32)).copy())
        for t in reversed(tapes):
            g.adjoint_step(t.data_ptr(), dt)
        out[adj] = (sum(float(np.sum(d[n] * get_adj(g, n))) for n in d), g.adjoint_tension(), g.adjoint_gravity())
        if adj == "fp32":
            with pytest.raises(SvofError, match="FP32"):
                g.adjoint_view("ifrcx")
        g.close()
    for a_, b_ in zip(out["fp32"], out["fp64"]):
        assert np.isfinite(a_) and rel(a_, b_) <= 1e-5, (out, a_, b_)
