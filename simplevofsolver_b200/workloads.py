"""Seeded synthetic initial conditions in the reference's restart (NPY) layout.

The reference reads its initial condition from a directory of NPY files
(``src/main.c:58-84``): ``step``, ``time``, ``glsizes`` (uint64), ``lengths``,
``xf`` (nx+1), ``xc`` (nx+2) and the fields ``ux`` (ny, nx+1) and ``uy``,
``p``, ``t``, ``vof`` (ny, nx+2), all float64 in C order, x fastest, x ghost
cells included and no y halo (``src/array.c:80-144``,
``initial_condition/main.py:46-73``).  This module builds such sets for the
droplet workloads; no dataset is involved, every input is generated from a
fixed seed.

Grids: a uniform x grid (``np.linspace``), or the tanh-stretched grid
``xf_i = lx * (1 + tanh(s (2 i / nx - 1)) / tanh(s)) / 2`` clustered at the
walls.  Cell centres follow the reference generator: ``xc = [0, midpoints,
lx]``.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class InitialCondition:
    nx: int
    ny: int
    lx: float
    ly: float
    xf: np.ndarray
    xc: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    p: np.ndarray
    t: np.ndarray
    vof: np.ndarray
    env: dict = field(default_factory=dict)

    def fields(self):
        return {"ux": self.ux, "uy": self.uy, "p": self.p, "t": self.t, "vof": self.vof}


def x_grid(nx: int, lx: float, uniform: bool = True, stretch: float = 1.5):
    if uniform:
        xf = np.linspace(0.0, lx, nx + 1, endpoint=True)
    else:
        s = float(stretch)
        i = np.arange(nx + 1, dtype=np.float64)
        xf = lx * 0.5 * (1.0 + np.tanh(s * (2.0 * i / nx - 1.0)) / np.tanh(s))
        xf[0] = 0.0
        xf[-1] = lx
    xc = np.concatenate(([0.0], 0.5 * xf[:-1] + 0.5 * xf[1:], [lx]))
    return xf.astype(np.float64), xc.astype(np.float64)


def _ellipse_distance(x, y, x0, y0, a, b):
    """First-order signed distance to the ellipse ((x-x0)/a)^2 + ((y-y0)/b)^2 = 1:
    (q - 1) / |grad q| with q the normalised radius (negative inside)."""
    X = x - x0
    Y = y - y0
    q = np.sqrt((X / a) ** 2 + (Y / b) ** 2)
    g = np.sqrt((X / a**2) ** 2 + (Y / b**2) ** 2) / np.maximum(q, 1e-300)
    return (q - 1.0) / np.maximum(g, 1e-300)


def droplet2d(nx: int = 128, ny: int = 128, lx: float = 1.0, ly: float = 1.0,
              uniform: bool = True, centre=(0.5, 0.5), semi_axes=(0.30, 0.20),
              noise: float = 1.0e-6, seed: int = 0, nsub: int = 8,
              stretch: float = 1.5) -> InitialCondition:
    """One elliptical droplet (vof = 1 inside) in a wall-bounded (x) and
    periodic (y) box.

    vof is the cell average of 0.5 (1 - tanh(phi / w)), w = h / 3 with h the
    nominal spacing lx / nx (a one-third-cell interface width), integrated by
    an nsub x nsub midpoint rule inside every cell.  The velocity is zero plus
    uniform white noise in [-noise, +noise] on the interior faces
    (``numpy.random.default_rng(seed)``); p and t are zero.
    """
    xf, xc = x_grid(nx, lx, uniform, stretch)
    dy = ly / ny
    w = (lx / nx) / 3.0
    # sub-cell sample points
    frac = (np.arange(nsub) + 0.5) / nsub
    xs = (xf[:-1, None] + np.diff(xf)[:, None] * frac[None, :]).reshape(-1)          # nx*nsub
    ys = ((np.arange(ny)[:, None] + frac[None, :]) * dy).reshape(-1)                 # ny*nsub
    X, Y = np.meshgrid(xs, ys, indexing="xy")                                         # (ny*nsub, nx*nsub)
    phi = _ellipse_distance(X, Y, centre[0], centre[1], semi_axes[0], semi_axes[1])
    h = 0.5 * (1.0 - np.tanh(phi / w))
    cellavg = h.reshape(ny, nsub, nx, nsub).mean(axis=(1, 3))
    vof = np.zeros((ny, nx + 2))
    vof[:, 1:-1] = cellavg
    rng = np.random.default_rng(seed)
    ux = np.zeros((ny, nx + 1))
    uy = np.zeros((ny, nx + 2))
    ux[:, 1:-1] = rng.uniform(-noise, noise, size=(ny, nx - 1))
    uy[:, 1:-1] = rng.uniform(-noise, noise, size=(ny, nx))
    p = np.zeros((ny, nx + 2))
    t = np.zeros((ny, nx + 2))
    return InitialCondition(nx, ny, lx, ly, xf, xc, ux, uy, p, t, vof)


@dataclass
class InitialCondition3D:
    """3D restart set: fields hold interior y and z rows and the x ghost
    cells: ux (nz, ny, nx+1); uy, uz, p, t, vof (nz, ny, nx+2)."""
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    xf: np.ndarray
    xc: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    uz: np.ndarray
    p: np.ndarray
    t: np.ndarray
    vof: np.ndarray
    env: dict = field(default_factory=dict)

    def fields(self):
        return {"ux": self.ux, "uy": self.uy, "uz": self.uz, "p": self.p, "t": self.t, "vof": self.vof}


def place_spheres(n: int, rmin: float, rmax: float, lx: float, ly: float, lz: float, wall_gap: float,
                  rng, gap: float = 0.0, max_tries: int = 200000):
    """Seeded rejection sampling of ``n`` non-overlapping spheres (radius
    uniform in [rmin, rmax]) at least ``wall_gap`` from the x walls; y and z
    are periodic, so distances use the minimum image."""
    out = []
    tries = 0
    while len(out) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could not place {n} spheres")
        r = rng.uniform(rmin, rmax)
        x = rng.uniform(r + wall_gap, lx - r - wall_gap)
        y = rng.uniform(0.0, ly)
        z = rng.uniform(0.0, lz)
        ok = True
        for (x2, y2, z2, r2) in out:
            dy = abs(y - y2)
            dy = min(dy, ly - dy)
            dz = abs(z - z2)
            dz = min(dz, lz - dz)
            if (x - x2) ** 2 + dy ** 2 + dz ** 2 < (r + r2 + gap) ** 2:
                ok = False
                break
        if ok:
            out.append((x, y, z, r))
    return out


def _sphere_vof(vof, xf, ny, nz, ly, lz, sphere, w, band, nsub):
    """Adds one sphere's cell-averaged 0.5 (1 - tanh(phi / w)) to ``vof``
    (nz, ny, nx+2): cells farther than ``band`` from the surface are 0 or 1
    exactly, the band cells are integrated by an nsub^3 midpoint rule."""
    x0, y0, z0, r = sphere
    nx = xf.size - 1
    dy, dz = ly / ny, lz / nz
    xcen = 0.5 * (xf[:-1] + xf[1:])
    i0 = max(int(np.searchsorted(xf, x0 - r - band)) - 1, 0)
    i1 = min(int(np.searchsorted(xf, x0 + r + band)) + 1, nx)
    j0 = int(np.floor((y0 - r - band) / dy)) - 1
    j1 = int(np.ceil((y0 + r + band) / dy)) + 1
    k0 = int(np.floor((z0 - r - band) / dz)) - 1
    k1 = int(np.ceil((z0 + r + band) / dz)) + 1
    ii = np.arange(i0, i1)
    jj = np.arange(j0, j1)
    kk = np.arange(k0, k1)
    X = xcen[ii][None, None, :]
    Y = ((jj + 0.5) * dy)[None, :, None]
    Z = ((kk + 0.5) * dz)[:, None, None]
    phi = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2 + (Z - z0) ** 2) - r
    inside = phi < -band
    near = np.abs(phi) <= band
    val = np.where(inside, 1.0, 0.0)
    kn, jn, in_ = np.nonzero(near)
    if kn.size:
        frac = (np.arange(nsub) + 0.5) / nsub
        dxc = (xf[1:] - xf[:-1])[ii[in_]]
        xs = xf[ii[in_]][:, None] + dxc[:, None] * frac[None, :]
        ys = (jj[jn][:, None] + frac[None, :]) * dy
        zs = (kk[kn][:, None] + frac[None, :]) * dz
        acc = np.zeros(kn.size)
        for a in range(nsub):
            d2 = (zs[:, a][:, None, None] - z0) ** 2 + (ys[:, :, None] - y0) ** 2 + \
                 (xs[:, None, :] - x0) ** 2
            ph = np.sqrt(d2) - r
            acc += (0.5 * (1.0 - np.tanh(ph / w))).sum(axis=(1, 2))
        val[kn, jn, in_] = acc / nsub ** 3
    jm = np.mod(jj, ny)
    km = np.mod(kk, nz)
    sub = vof[np.ix_(km, jm, ii + 1)]
    vof[np.ix_(km, jm, ii + 1)] = np.maximum(sub, val)


def random_potential(ny, nz, ly, lz, kmax, rng):
    """Coefficients of one random Fourier potential: a list of
    (ky, kz, amplitude, phase) with 0 < ky^2 + kz^2 <= kmax^2, amplitudes
    standard normal over |k|"""
    modes = []
    for ky in range(-kmax, kmax + 1):
        for kz in range(-kmax, kmax + 1):
            if ky * ky + kz * kz == 0 or ky * ky + kz * kz > kmax * kmax:
                continue
            modes.append((ky, kz, rng.standard_normal() / np.hypot(ky, kz), rng.uniform(0.0, 2.0 * np.pi)))
    return modes


def eval_potential(modes, ny, nz, ly, lz, yoff, zoff):
    y = (np.arange(ny) + yoff) * (ly / ny)
    z = (np.arange(nz) + zoff) * (lz / nz)
    out = np.zeros((nz, ny))
    for ky, kz, a, th in modes:
        out += a * np.cos(2.0 * np.pi * (ky * y[None, :] / ly + kz * z[:, None] / lz) + th)
    return out


def droplets3d(nx: int = 256, ny: int = 256, nz: int = 256, lx: float = 1.0, ly: float = 1.0,
               lz: float = 1.0, uniform: bool = False, stretch: float = 1.5, ndrops: int = 32,
               radii=(0.04, 0.08), urms: float = 0.5, kmax: int = 4, seed: int = 1, nsub: int = 4,
               velocity: bool = True) -> InitialCondition3D:
    """Spherical droplets in a wall-bounded (x), doubly periodic (y, z) box.

    * Spheres: ``place_spheres`` with radii uniform in ``radii``, no overlap,
      at least two nominal cells from the walls (``numpy.random.default_rng(seed)``).
    * vof: cell average of 0.5 (1 - tanh(phi / w)), phi the distance to the
      sphere surface, w = (lx / nx) / 3; cells within 8 w of a surface by an
      nsub^3 midpoint rule, the rest exactly 0 or 1.
    * Velocity: the staggered discrete curl of A = (0, f(x) a(y, z), f(x) b(y, z)),
      f = sin^2(pi x / lx) (zero with its slope at the walls, so ux vanishes
      there), a and b random Fourier sums over 0 < |k| <= kmax: ux = f (db/dy
      - da/dz), uy = -(df/dx) b, uz = (df/dx) a, differenced on the grid so
      the discrete divergence vanishes to round-off; scaled so that
      sqrt(mean(ux^2 + uy^2 + uz^2) / 3) = urms.  p and t are zero.
    """
    rng = np.random.default_rng(seed)
    xf, xc = x_grid(nx, lx, uniform, stretch)
    h = lx / nx
    w = h / 3.0
    spheres = place_spheres(ndrops, radii[0], radii[1], lx, ly, lz, 2.0 * h, rng)
    vof = np.zeros((nz, ny, nx + 2))
    for sp in spheres:
        _sphere_vof(vof, xf, ny, nz, ly, lz, sp, w, 8.0 * w, nsub)
    ux = np.zeros((nz, ny, nx + 1))
    uy = np.zeros((nz, ny, nx + 2))
    uz = np.zeros((nz, ny, nx + 2))
    if velocity and urms > 0.0:
        dy, dz = ly / ny, lz / nz
        ma = random_potential(ny, nz, ly, lz, kmax, rng)
        mb = random_potential(ny, nz, ly, lz, kmax, rng)
        # Ay on (x face, y centre, z face), Az on (x face, y face, z centre)
        a = eval_potential(ma, ny, nz, ly, lz, 0.5, 0.0)
        b = eval_potential(mb, ny, nz, ly, lz, 0.0, 0.5)
        f = np.sin(np.pi * xf / lx) ** 2                       # at x faces, f(0) = f(lx) = 0
        f[0] = 0.0
        f[-1] = 0.0
        # ux at (x face i, y centre j, z centre k): dAz/dy - dAy/dz
        dbdy = (np.roll(b, -1, axis=1) - b) / dy               # (nz, ny): b(j+1) - b(j)
        dadz = (np.roll(a, -1, axis=0) - a) / dz
        ux[...] = f[None, None, :] * (dbdy - dadz)[:, :, None]
        # uy at (x centre, y face j, z centre): -dAz/dx; uz at (x centre, y centre, z face k): dAy/dx
        dfdx = (f[1:] - f[:-1]) / (xf[1:] - xf[:-1])           # (nx,)
        uy[:, :, 1:-1] = -dfdx[None, None, :] * b[:, :, None]
        uz[:, :, 1:-1] = dfdx[None, None, :] * a[:, :, None]
        rms = np.sqrt((np.mean(ux[:, :, 1:-1] ** 2) + np.mean(uy[:, :, 1:-1] ** 2) +
                       np.mean(uz[:, :, 1:-1] ** 2)) / 3.0)
        s = urms / rms
        ux *= s
        uy *= s
        uz *= s
    p = np.zeros((nz, ny, nx + 2))
    t = np.zeros((nz, ny, nx + 2))
    ic = InitialCondition3D(nx, ny, nz, lx, ly, lz, xf, xc, ux, uy, uz, p, t, vof)
    ic.spheres = spheres
    return ic


def extrude_z(ic: InitialCondition, nz: int, lz: float = 1.0) -> InitialCondition3D:
    """A 2D set repeated along z (uz = 0): the 3D solver on it reproduces the
    2D solver."""
    rep = lambda a: np.ascontiguousarray(np.broadcast_to(a[None], (nz,) + a.shape))
    return InitialCondition3D(ic.nx, ic.ny, nz, ic.lx, ic.ly, lz, ic.xf.copy(), ic.xc.copy(),
                              rep(ic.ux), rep(ic.uy), np.zeros((nz, ic.ny, ic.nx + 2)), rep(ic.p),
                              rep(ic.t), rep(ic.vof))


def extrude_y(ic: InitialCondition, ny: int, ly: float = 1.0) -> InitialCondition3D:
    """A 2D set laid in the x-z plane and repeated along y (uy = 0, the 2D
    y velocity becomes uz)."""
    rep = lambda a: np.ascontiguousarray(np.broadcast_to(a[:, None, :], (a.shape[0], ny, a.shape[1])))
    return InitialCondition3D(ic.nx, ny, ic.ny, ic.lx, ly, ic.ly, ic.xf.copy(), ic.xc.copy(),
                              rep(ic.ux), np.zeros((ic.ny, ny, ic.nx + 2)), rep(ic.uy), rep(ic.p),
                              rep(ic.t), rep(ic.vof))


# Environment of the 3D droplet workloads: Re = 500 (m_dif = 1 / Re through
# Ra = 2.5e5, Pr = 1), We = 20, CFL safety 0.5.
DROPLETS3D_ENV = {"Ra": 2.5e5, "Pr": 1.0, "We": 20.0, "coef_dt_adv": 0.5, "coef_dt_dif": 0.95}


# Environment of the 2D droplet workload: Re = sqrt(Ra)/sqrt(Pr) = 100 gives
# nu = m_dif = 0.01, We = 10, CFL safety 0.5 (src/fluid/init.c:90-93,
# src/interface/init.c:66-68, src/fluid/decide_dt.c:109-112).
DROPLET2D_ENV = {"Ra": 1.0e4, "Pr": 1.0, "We": 10.0, "coef_dt_adv": 0.5, "coef_dt_dif": 0.95}


# the falling droplet of the differentiation workload: Re = 200 (Ra = Re^2 with
# Pr = 1 gives m_dif = 1 / Re), We = 20; gravity Fr = 1 and the density ratio
# 0.1 enter as the vof buoyancy coefficient grav_vof = -(1 - 0.1) / Fr^2
FALLING2D_ENV = {"Ra": 4.0e4, "Pr": 1.0, "We": 20.0, "coef_dt_adv": 0.5, "coef_dt_dif": 0.95}
FALLING2D_FROUDE = 1.0
FALLING2D_DENSITY_RATIO = 0.1


def falling_droplet2d(n: int = 256, radius: float = 0.15, centre=(0.5, 0.7), rms: float = 0.05,
                      kmax: int = 3, seed: int = 0, uniform: bool = True) -> InitialCondition:
    """One circular droplet (radius 0.15 at (0.5, 0.7)) in the unit box, and a
    seeded divergence-free random velocity of the given rms: the staggered
    curl of the stream function sin^2(pi x) sum_k (a_k cos 2 pi k y + b_k
    sin 2 pi k y), 1 <= k <= kmax, evaluated at the cell corners, so that the
    discrete divergence vanishes and ux vanishes at the walls.  vof as
    droplet2d (tanh profile of one-third-cell width, sub-cell integration)."""
    ic = droplet2d(n, n, 1.0, 1.0, uniform=uniform, centre=centre, semi_axes=(radius, radius), noise=0.0,
                   seed=seed)
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(kmax)
    b = rng.standard_normal(kmax)
    yf = np.arange(n + 1) * (1.0 / n)                                 # corner rows y_{j-1/2}
    xf = ic.xf
    k = np.arange(1, kmax + 1)[:, None]
    fy = (a[:, None] * np.cos(2 * np.pi * k * yf[None, :]) + b[:, None] * np.sin(2 * np.pi * k * yf[None, :])).sum(0)
    psi = (np.sin(np.pi * xf) ** 2)[None, :] * fy[:, None]            # (n+1 corners in y, n+1 in x)
    dy = 1.0 / n
    dxf = np.diff(xf)
    ux = (psi[1:, :] - psi[:-1, :]) / dy                              # (n, n+1) faces, rows j
    uy = -(psi[:, 1:] - psi[:, :-1]) / dxf[None, :]                   # (n+1, n) rows j-1/2
    scale = rms / np.sqrt(0.5 * (np.mean(ux[:, 1:-1] ** 2) + np.mean(uy ** 2)))
    ic.ux[:, 1:-1] = scale * ux[:, 1:-1]
    ic.uy[:, 1:-1] = scale * uy[:-1, :]
    return ic


def falling_gravity(ic: InitialCondition, froude: float = FALLING2D_FROUDE,
                    density_ratio: float = FALLING2D_DENSITY_RATIO):
    """(grav_vof, vof_ref) of the vof buoyancy extension: gravity -1/Fr^2
    along y on the density difference (1 - ratio) vof, relative to the
    domain-mean volume fraction (no net force along the periodic y)"""
    dxf = np.diff(ic.xf)
    vof_ref = float(np.sum(ic.vof[:, 1:-1] * dxf[None, :]) / (ic.ly * ic.lx) * (ic.ly / ic.ny))
    return -(1.0 - density_ratio) / froude ** 2, vof_ref


# The 3D differentiation workload: the 3D generator at n^3 (stretched x) with
# 16 droplets of radii in [0.05, 0.09], the 3D environment (Re = 500, We =
# 20), the vof buoyancy extension with density ratio 0.05 at Fr = 1 (gravity
# along -y), 100 steps.
DIFF3D_DENSITY_RATIO = 0.05
DIFF3D_FROUDE = 1.0


def diff3d_case(n: int = 256, seed: int = 1) -> InitialCondition3D:
    return droplets3d(n, n, n, ndrops=16, radii=(0.05, 0.09), seed=seed)


def gravity3d(ic: InitialCondition3D, froude: float = DIFF3D_FROUDE,
              density_ratio: float = DIFF3D_DENSITY_RATIO):
    """(grav_vof, vof_ref) of the 3D vof buoyancy extension: gravity -1/Fr^2
    along y on the density difference (1 - ratio) vof, relative to the
    domain-mean volume fraction (no net force along the periodic y);
    d grav_vof / d ratio = 1 / Fr^2"""
    dxf = np.diff(ic.xf)
    vof_ref = float(np.sum(ic.vof[..., 1:-1] * dxf) / (ic.lx * ic.ny * ic.nz))
    return -(1.0 - density_ratio) / froude ** 2, vof_ref


def physical_params(env: dict):
    """Diffusivities and surface tension as the reference derives them."""
    Ra, Pr, We = float(env["Ra"]), float(env["Pr"]), float(env["We"])
    m_dif = 1.0 * np.sqrt(Pr) / np.sqrt(Ra)
    t_dif = 1.0 / np.sqrt(Pr) / np.sqrt(Ra)
    return dict(m_dif=float(m_dif), t_dif=float(t_dif), tension=float(1.0 / We),
                coef_dt_adv=float(env["coef_dt_adv"]), coef_dt_dif=float(env["coef_dt_dif"]))


def write_npy_dir(ic, dirname: str, step: int = 0, time: float = 0.0):
    """a restart directory in the reference's layout (src/main.c:64-71,
    src/domain.c:60-74, src/fluid/save.c, src/interface/save.c): step, time,
    glsizes, lengths, xf, xc and the fields' interior rows with their x ghost
    cells; 2D (InitialCondition) or 3D (InitialCondition3D: one more size and
    length, uz)"""
    os.makedirs(dirname, exist_ok=True)
    three = hasattr(ic, "nz")
    sizes = [ic.nx, ic.ny, ic.nz] if three else [ic.nx, ic.ny]
    lengths = [ic.lx, ic.ly, ic.lz] if three else [ic.lx, ic.ly]
    np.save(os.path.join(dirname, "step.npy"), np.array(step, dtype=np.uint64))
    np.save(os.path.join(dirname, "time.npy"), np.array(time, dtype=np.float64))
    np.save(os.path.join(dirname, "glsizes.npy"), np.array(sizes, dtype=np.uint64))
    np.save(os.path.join(dirname, "lengths.npy"), np.array(lengths, dtype=np.float64))
    np.save(os.path.join(dirname, "xf.npy"), ic.xf.astype(np.float64))
    np.save(os.path.join(dirname, "xc.npy"), ic.xc.astype(np.float64))
    for k, v in ic.fields().items():
        np.save(os.path.join(dirname, f"{k}.npy"), np.ascontiguousarray(v, dtype=np.float64))


def _load_npy(dirname: str, name: str, shape=None, dtype=np.float64):
    """one array of a restart directory, checked against the reference's
    layout (little-endian, C order, the given dtype and shape); a file that
    is not a readable NPY v1/v2 array, or that differs, raises ValueError
    naming the file"""
    path = os.path.join(dirname, f"{name}.npy")
    try:
        a = np.load(path, allow_pickle=False)
    except (ValueError, OSError, EOFError) as e:
        raise ValueError(f"{path}: not a readable NPY array ({e})") from None
    want = np.dtype(dtype).newbyteorder("<")
    if a.dtype != want:
        raise ValueError(f"{path}: dtype {a.dtype.str}, expected {want.str}")
    if a.ndim > 1 and not a.flags.c_contiguous:
        raise ValueError(f"{path}: Fortran order, expected C order")
    if shape is not None and tuple(a.shape) != tuple(shape):
        raise ValueError(f"{path}: shape {tuple(a.shape)}, expected {tuple(shape)}")
    return a


def read_npy_dir(dirname: str):
    """the restart directory written by write_npy_dir or by the reference's
    save: InitialCondition (2D) or InitialCondition3D (glsizes of 3 items).
    Every array is checked against the reference's layout (float64 fields
    with the x ghost cells: ux (.., nx + 1), the others (.., nx + 2); xf of
    nx + 1, xc of nx + 2 values; uint64 glsizes): ValueError otherwise."""
    gl = _load_npy(dirname, "glsizes", None, np.uint64)
    if gl.ndim != 1 or len(gl) not in (2, 3) or np.any(gl < 1):
        raise ValueError(f"{dirname}: glsizes {gl.tolist()} is not a 2D or 3D grid size")
    ln = _load_npy(dirname, "lengths", (len(gl),))
    nx = int(gl[0])
    xf = _load_npy(dirname, "xf", (nx + 1,))
    xc = _load_npy(dirname, "xc", (nx + 2,))
    rows = tuple(int(v) for v in gl[1:][::-1])  # (ny,) or (nz, ny)
    fx, fc = rows + (nx + 1,), rows + (nx + 2,)
    ld = lambda k: _load_npy(dirname, k, fx if k == "ux" else fc)
    if 3 == len(gl):
        ny, nz = int(gl[1]), int(gl[2])
        return InitialCondition3D(nx, ny, nz, float(ln[0]), float(ln[1]), float(ln[2]), xf, xc,
                                  ld("ux"), ld("uy"), ld("uz"), ld("p"), ld("t"), ld("vof"))
    ny = int(gl[1])
    return InitialCondition(nx, ny, float(ln[0]), float(ln[1]), xf, xc,
                            ld("ux"), ld("uy"), ld("p"), ld("t"), ld("vof"))
