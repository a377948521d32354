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


# Environment of the 2D droplet workload: Re = sqrt(Ra)/sqrt(Pr) = 100 gives
# nu = m_dif = 0.01, We = 10, CFL safety 0.5 (src/fluid/init.c:90-93,
# src/interface/init.c:66-68, src/fluid/decide_dt.c:109-112).
DROPLET2D_ENV = {"Ra": 1.0e4, "Pr": 1.0, "We": 10.0, "coef_dt_adv": 0.5, "coef_dt_dif": 0.95}


def physical_params(env: dict):
    """Diffusivities and surface tension as the reference derives them."""
    Ra, Pr, We = float(env["Ra"]), float(env["Pr"]), float(env["We"])
    m_dif = 1.0 * np.sqrt(Pr) / np.sqrt(Ra)
    t_dif = 1.0 / np.sqrt(Pr) / np.sqrt(Ra)
    return dict(m_dif=float(m_dif), t_dif=float(t_dif), tension=float(1.0 / We),
                coef_dt_adv=float(env["coef_dt_adv"]), coef_dt_dif=float(env["coef_dt_dif"]))


def write_npy_dir(ic: InitialCondition, dirname: str, step: int = 0, time: float = 0.0):
    os.makedirs(dirname, exist_ok=True)
    np.save(os.path.join(dirname, "step.npy"), np.array(step, dtype=np.uint64))
    np.save(os.path.join(dirname, "time.npy"), np.array(time, dtype=np.float64))
    np.save(os.path.join(dirname, "glsizes.npy"), np.array([ic.nx, ic.ny], dtype=np.uint64))
    np.save(os.path.join(dirname, "lengths.npy"), np.array([ic.lx, ic.ly], dtype=np.float64))
    np.save(os.path.join(dirname, "xf.npy"), ic.xf.astype(np.float64))
    np.save(os.path.join(dirname, "xc.npy"), ic.xc.astype(np.float64))
    for k, v in ic.fields().items():
        np.save(os.path.join(dirname, f"{k}.npy"), np.ascontiguousarray(v, dtype=np.float64))


def read_npy_dir(dirname: str) -> InitialCondition:
    ld = lambda k: np.load(os.path.join(dirname, f"{k}.npy"))
    gl = ld("glsizes")
    ln = ld("lengths")
    nx, ny = int(gl[0]), int(gl[1])
    return InitialCondition(nx, ny, float(ln[0]), float(ln[1]), ld("xf"), ld("xc"),
                            ld("ux"), ld("uy"), ld("p"), ld("t"), ld("vof"))
