"""The 3D restatement (oracle/svof_oracle3d.c) against the pinned 2D one.

The mounted reference is its 2D branch, so the 3D restatement cannot be run
against reference output.  It is pinned instead through two reductions: a 2D
field repeated along z (uz = 0) and a 2D field laid in the x-z plane and
repeated along y (uy = 0, the 2D y velocity becomes uz).  In both, every 3D
function must reproduce the pinned 2D function.  Each function is compared
from the same synchronised state.  Differences may come only from summation
order: the 8-point THINC sums against the 4-point ones, and the corner-gradient
scale at the ``1/max(|g|, DBL_EPSILON)`` clamp of vanishing gradients, where
the force is ~0.  The momentum predictor, the Poisson solve (gauge mean
removed), the projection and the pressure update must be bit-identical.
"""
import numpy as np
import pytest

from oracle import Oracle, Oracle3D
from simplevofsolver_b200.workloads import (DROPLET2D_ENV, DROPLETS3D_ENV, droplet2d, droplets3d, extrude_y,
                                            extrude_z, physical_params)

STATE2D = ["ux", "uy", "p", "psi", "t", "vof", "curv", "srcux0", "srcux1", "srcuy0", "srcuy1", "srct0",
           "srct1", "src0", "src1", "ifrcx", "ifrcy"]
# per-function bound on max |3D - 2D| / max |2D| (p is compared modulo its mean,
# and the two means are summed over differently shaped arrays)
TOL = {"geom": 1e-11, "vof": 1e-15, "predict": 0.0, "potential": 1e-14, "correct": 0.0, "pressure": 1e-15}


class Pair:
    """a 2D oracle and a 3D oracle on its extrusion along ``axis``"""

    def __init__(self, ic2, axis, n3=4):
        prm = physical_params(DROPLET2D_ENV)
        self.axis = axis
        self.o2 = Oracle(ic2, prm)
        ic3 = extrude_z(ic2, n3) if axis == "z" else extrude_y(ic2, n3)
        self.o3 = Oracle3D(ic3, prm)
        self.map = {} if axis == "z" else {"uy": "uz", "srcuy0": "srcuz0", "srcuy1": "srcuz1", "ifrcy": "ifrcz"}
        self.zero = (["uz", "srcuz0", "srcuz1", "ifrcz"] if axis == "z" else
                     ["uy", "srcuy0", "srcuy1", "ifrcy"])

    def f3(self, k):
        return self.o3.field(self.map.get(k, k))

    def spread(self, a, shape3):
        return np.broadcast_to(a[None] if self.axis == "z" else a[:, None], shape3)

    def sync(self):
        for k in STATE2D:
            b = self.f3(k)
            b[...] = self.spread(self.o2.field(k), b.shape)
        for k in self.zero:
            self.o3.field(k)[...] = 0.0

    def diff(self, k):
        a = self.o2.field(k)
        b = self.f3(k)
        h = 2 if k == "vof" else (0 if k.startswith(("src", "ifrc")) else 1)
        if self.axis == "z":
            b = b[h:b.shape[0] - h] if h else b
            a3 = a[None]
        else:
            b = b[:, h:b.shape[1] - h] if h else b
            a3 = a[:, None]
        if k in ("p", "psi"):
            # modulo the round-off-fixed gauge constant, on the interior x
            # cells (the halo corner cells keep the previous call's values)
            a3 = (a3 - a[1:-1, 1:-1].mean())[..., 1:-1]
            b = (b - (b[:, 1:-1, 1:-1].mean() if self.axis == "z" else b[1:-1, :, 1:-1].mean()))[..., 1:-1]
        return np.abs(b - a3).max() / max(np.abs(a).max(), 1e-300)


def _per_function(pair, dt):
    o2, o3 = pair.o2, pair.o3
    worst = {}
    for rk in range(3):
        steps = [
            ("geom", lambda o: (o.curvature_tensor(), o.force()), ["ifrcx", "ifrcy"]),
            ("vof", lambda o: o.update_vof(rk, dt), ["vof", "src0"]),
            ("predict", lambda o: o.predict(rk, dt), ["ux", "uy", "t", "srcux0", "srcuy0", "srct0"]),
            ("potential", lambda o: o.potential(rk, dt), ["psi"]),
            ("correct", lambda o: o.correct(rk, dt), ["ux", "uy"]),
            ("pressure", lambda o: o.update_pressure(rk, dt), ["p"]),
        ]
        for name, fn, outs in steps:
            pair.sync()
            fn(o2)
            fn(o3)
            for k in outs:
                worst[(name, k)] = max(worst.get((name, k), 0.0), pair.diff(k))
        # advance the 2D state by the real substep for the next rk
        o2.curvature_tensor()
        o2.force()
        o2.update_vof(rk, dt)
        o2.predict(rk, dt)
        o2.potential(rk, dt)
        o2.correct(rk, dt)
        o2.update_pressure(rk, dt)
    return worst


@pytest.mark.parametrize("axis", ["z", "y"])
@pytest.mark.parametrize("uniform", [False, True])
def test_every_function_reduces_to_2d(axis, uniform):
    ic2 = droplet2d(32, 24, uniform=uniform, noise=1e-2)
    pair = Pair(ic2, axis)
    dt = pair.o2.decide_dt()
    worst = _per_function(pair, dt)
    for (name, k), d in worst.items():
        assert d <= TOL[name], (axis, name, k, d)


@pytest.mark.parametrize("axis", ["z", "y"])
def test_steps_reduce_to_2d(axis):
    """ten full steps with the 2D dt (the explicit diffusive dt limits
    differ with the number of dimensions)"""
    ic2 = droplet2d(32, 24, uniform=False, noise=1e-2)
    pair = Pair(ic2, axis)
    for _ in range(10):
        dt = pair.o2.decide_dt()
        for rk in range(3):
            for o in (pair.o2, pair.o3):
                o.curvature_tensor()
                o.force()
                o.update_vof(rk, dt)
                o.predict(rk, dt)
                o.potential(rk, dt)
                o.correct(rk, dt)
                o.update_pressure(rk, dt)
    for k in ("ux", "uy", "vof", "p"):
        assert pair.diff(k) <= 1e-11, (axis, k, pair.diff(k))
    assert np.abs(pair.o3.field(pair.zero[0])).max() == 0.0


def test_decide_dt_uses_three_dimensions():
    """the explicit diffusive limit is coef/nu * 0.5 / NDIMS * dy^2 with NDIMS = 3"""
    ic2 = droplet2d(32, 24, uniform=False, noise=0.0)
    pair = Pair(ic2, "z")
    prm = physical_params(DROPLET2D_ENV)
    dy = 1.0 / 24
    want = min(prm["coef_dt_dif"] / prm["m_dif"] * 0.5 / 3 * dy**2,
               prm["coef_dt_dif"] / prm["t_dif"] * 0.5 / 3 * dy**2,
               prm["coef_dt_adv"] * 1.0)
    assert pair.o3.decide_dt() == pytest.approx(want, rel=1e-15)


def _divergence(o, ic):
    dxf = np.diff(ic.xf)
    dy, dz = ic.ly / ic.ny, ic.lz / ic.nz
    ux = o.field("ux")[1:-1, 1:-1]
    uy = o.field("uy")[1:-1]
    uz = o.field("uz")
    return ((ux[:, :, 1:] - ux[:, :, :-1]) / dxf + (uy[:, 2:, 1:-1] - uy[:, 1:-1, 1:-1]) / dy +
            (uz[2:, 1:-1, 1:-1] - uz[1:-1, 1:-1, 1:-1]) / dz)


def test_droplets3d_projection_and_volume():
    """a genuinely 3D field: projected velocity is divergence-free and the
    flux-form vof update conserves volume"""
    ic = droplets3d(24, 16, 20, ndrops=3, radii=(0.12, 0.2), seed=3)
    o = Oracle3D(ic, physical_params(DROPLETS3D_ENV))
    dxf = np.diff(ic.xf)

    def volume():
        return float(np.sum(o.field("vof")[2:-2, 2:-2, 1:-1] * dxf)) * (ic.ly / ic.ny) * (ic.lz / ic.nz)

    v0 = volume()
    dts = o.run(5)
    assert np.all(dts > 0)
    assert np.abs(_divergence(o, ic)).max() < 1e-11
    assert abs(volume() - v0) / v0 < 1e-13
    v = o.field("vof")
    assert v.min() > -1e-3 and v.max() < 1 + 1e-3


def test_generator_is_divergence_free_and_seeded():
    a = droplets3d(32, 16, 24, ndrops=4, radii=(0.1, 0.15), seed=5)
    b = droplets3d(32, 16, 24, ndrops=4, radii=(0.1, 0.15), seed=5)
    for k, v in a.fields().items():
        assert np.array_equal(v, b.fields()[k]), k
    dxf = np.diff(a.xf)
    ux, uy, uz = a.ux, a.uy[:, :, 1:-1], a.uz[:, :, 1:-1]
    div = ((ux[:, :, 1:] - ux[:, :, :-1]) / dxf + (np.roll(uy, -1, axis=1) - uy) * a.ny +
           (np.roll(uz, -1, axis=0) - uz) * a.nz)
    assert np.abs(div).max() < 1e-11 * max(np.abs(ux).max(), 1.0) * a.nx
    assert np.all(a.ux[:, :, 0] == 0) and np.all(a.ux[:, :, -1] == 0)
    rms = np.sqrt((np.mean(ux[:, :, 1:-1] ** 2) + np.mean(uy ** 2) + np.mean(uz ** 2)) / 3)
    assert rms == pytest.approx(0.5, rel=1e-12)
    # spheres do not overlap (periodic y, z) and keep two cells from the walls
    sp = a.spheres
    for m, (x, y, z, r) in enumerate(sp):
        assert x - r >= 2.0 / a.nx and x + r <= 1.0 - 2.0 / a.nx
        for (x2, y2, z2, r2) in sp[m + 1:]:
            dy = min(abs(y - y2), 1 - abs(y - y2))
            dz = min(abs(z - z2), 1 - abs(z - z2))
            assert (x - x2) ** 2 + dy ** 2 + dz ** 2 >= (r + r2) ** 2


def test_vof_buoyancy_term_is_the_last_addition():
    """the extension adds grav (0.5 vof(j-1) + 0.5 vof(j) - vof_ref) to uy's
    src_a after every reference term: the source with it on equals the source
    without it plus the term, bit for bit; grav 0 leaves the step unchanged"""
    ic = droplets3d(24, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    a, b = Oracle3D(ic, phys), Oracle3D(ic, phys)
    b.set_gravity(-0.9, 0.2)
    dt = a.decide_dt()
    for o in (a, b):
        o.curvature_tensor()
        o.force()
        o.update_vof(0, dt)
        o.predict(0, dt)
    vof = b.field("vof")                                     # after the advection
    nz, ny, nx = 16, 16, 24
    v = vof[2:nz + 2, :, 1:nx + 1]                           # rows j = -1 .. ny+2 at index j + 1
    face = 0.5 * v[:, 0 + 1:ny + 1] + 0.5 * v[:, 1 + 1:ny + 2] - 0.2
    expect = a.field("srcuy0") + (-0.9) * face
    assert np.array_equal(b.field("srcuy0"), expect)
    c = Oracle3D(ic, phys)
    c.set_gravity(0.0, 0.7)
    a2 = Oracle3D(ic, phys)
    c.run(2)
    a2.run(2)
    for k in ("ux", "uy", "uz", "p", "vof"):
        assert np.array_equal(c.field(k), a2.field(k))
