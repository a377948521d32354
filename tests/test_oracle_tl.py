"""The oracle's tangent-linear model (oracle/svof_oracle_tl.inc) against
central finite differences of the oracle's own forward step.

The tangent model is the checker of the CUDA adjoint (the dot-product test
in test_gpu_adjoint.py); here it is itself pinned to the primal functions it
linearises.  The time step is held fixed in both.  A random weight w defines
J(x) = <w, F(x)> over the final ux, uy, p and vof (the weights of p sum to
zero: its additive constant is fixed by round-off); the directional derivative
of J along a random direction of unit norm (initial velocities, vof of
interfacial cells, surface tension, the vof buoyancy coefficient where it is
on) from the tangent model must match
(J(x + eps v) - J(x - eps v)) / (2 eps), eps = 1e-6, to 1e-7 relative.
"""
import numpy as np
import pytest

from oracle import Oracle
from simplevofsolver_b200.workloads import DROPLET2D_ENV, droplet2d, physical_params

INTERIOR = {"ux": (1, 1), "uy": (1, 1), "p": (1, 1), "vof": (2, 1)}  # halo rows, x ghost offset


def interior(name, a, nx, ny):
    h, _ = INTERIOR[name]
    if name == "ux":
        return a[h:h + ny, 1:nx]          # interior faces i = 2 .. nx
    return a[h:h + ny, 1:nx + 1]


def make(ic, phys, gravity=None):
    o = Oracle(ic, phys)
    if gravity:
        o.set_gravity(*gravity)
    return o


def perturbed(ic, phys, v, eps, gravity=None, dtension=0.0, dgrav=0.0):
    p = dict(phys)
    p["tension"] = phys["tension"] + eps * dtension
    o = make(ic, p, (gravity[0] + eps * dgrav, gravity[1]) if gravity else None)
    for k in ("ux", "uy", "vof"):
        interior(k, o.field(k), o.nx, o.ny)[...] += eps * v[k]
    import oracle
    oracle._load().svo_init_boundaries(o._h)
    return o


def objective(o, w):
    return sum(float(np.sum(w[k] * interior(k, o.field(k), o.nx, o.ny))) for k in w)


def directions(ic, o, seed):
    rng = np.random.default_rng(seed)
    nx, ny = o.nx, o.ny
    vof = interior("vof", o.field("vof"), nx, ny)
    inter = (vof > 1e-6) & (vof < 1 - 1e-6)
    v = {"ux": rng.standard_normal((ny, nx - 1)), "uy": rng.standard_normal((ny, nx)),
         "vof": rng.standard_normal((ny, nx)) * inter * 1e-2}
    w = {k: rng.standard_normal(s) for k, s in (("ux", (ny, nx - 1)), ("uy", (ny, nx)), ("p", (ny, nx)),
                                                 ("vof", (ny, nx)))}
    # unit L2 norm over all entries: with eps = 1e-6 each entry moves by
    # ~1e-8, well inside the range where the THINC geometry is linear (its
    # nonlinearity sets in at ~1e-4 near small interface gradients)
    nrm = np.sqrt(sum(float(np.sum(a * a)) for a in v.values()))
    v = {k: a / nrm for k, a in v.items()}
    # the pressure's additive constant is fixed by round-off: weights of p
    # sum to zero so that J does not see it
    w["p"] -= w["p"].mean()
    return v, w


@pytest.mark.parametrize("uniform,gravity,steps", [(True, None, 1), (False, None, 1), (True, (-0.9, 0.1), 3),
                                                   (False, (-0.9, 0.1), 3)])
def test_tangent_matches_central_differences(uniform, gravity, steps):
    ic = droplet2d(32, 32, uniform=uniform, noise=1e-2, semi_axes=(0.25, 0.2))
    phys = physical_params(DROPLET2D_ENV)
    base = make(ic, phys, gravity)
    dt = base.decide_dt()
    v, w = directions(ic, base, 7)
    dten = 0.3
    dgrav = 0.4 if gravity else 0.0
    # tangent: primal and tangent advanced together
    tan = base.tangent()
    for k in ("ux", "uy", "vof"):
        interior(k, tan.field(k), tan.nx, tan.ny)[...] = v[k]
    tan.init_boundaries()
    for _ in range(steps):
        tan.step(dt, dten, dgrav)
    dj_tl = sum(float(np.sum(w[k] * interior(k, tan.field(k), tan.nx, tan.ny))) for k in w)
    # central differences of the primal
    eps = 1e-6
    js = []
    for sgn in (+1, -1):
        o = perturbed(ic, phys, v, sgn * eps, gravity, dten, dgrav)
        for _ in range(steps):
            o.integrate_fixed(dt)
        js.append(objective(o, w))
    dj_fd = (js[0] - js[1]) / (2 * eps)
    assert abs(dj_fd - dj_tl) <= 1e-7 * abs(dj_tl), (dj_fd, dj_tl)


def test_tangent_is_linear():
    """doubling the direction doubles the tangent (no primal leaks into it)"""
    ic = droplet2d(32, 32, uniform=False, noise=1e-2)
    phys = physical_params(DROPLET2D_ENV)
    out = []
    for scale in (1.0, 2.0):
        base = make(ic, phys)
        dt = 1e-3
        v, _ = directions(ic, base, 3)
        tan = base.tangent()
        for k in ("ux", "uy", "vof"):
            interior(k, tan.field(k), tan.nx, tan.ny)[...] = scale * v[k]
        tan.init_boundaries()
        tan.step(dt, 0.1 * scale)
        out.append(np.concatenate([interior(k, tan.field(k), tan.nx, tan.ny).ravel() for k in ("ux", "uy", "vof")]))
    np.testing.assert_allclose(out[1], 2 * out[0], rtol=1e-13, atol=1e-13 * np.abs(out[1]).max())


def test_gravity_off_is_the_reference_step():
    """with the buoyancy coefficient zero the extension leaves the step
    bit-identical to the pinned one"""
    ic = droplet2d(32, 32, uniform=True, noise=1e-2)
    phys = physical_params(DROPLET2D_ENV)
    a = make(ic, phys)
    b = make(ic, phys, (0.0, 0.3))
    dt = a.decide_dt()
    for o in (a, b):
        o.integrate_fixed(dt)
        o.integrate_fixed(dt)
    for k in ("ux", "uy", "p", "vof"):
        assert np.array_equal(a.field(k), b.field(k)), k
    c = make(ic, phys)
    c.run(2)
    # integrate_fixed with the dt the CFL decision picks is integrate()
    e = make(ic, phys)
    for _ in range(2):
        e.integrate_fixed(e.decide_dt())
    for k in ("ux", "uy", "p", "vof"):
        assert np.array_equal(c.field(k), e.field(k)), k
