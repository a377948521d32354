"""One step on grids at the edges of the launch plans, against the oracle.

The parity tests use a few mid-size grids. The kernels' tiles, line lengths
and shared-memory plans change with the grid, and so do their edge cases:
- the smallest and largest FFT lengths (4 and 2048);
- odd and non-power-of-two sizes in the non-FFT directions;
- rows narrower than one tile;
- long, thin grids.

Each case runs one step through the C ABI and compares it with the oracle,
within the stated 1e-12 (p and psi modulo their mean).
"""
import numpy as np
import pytest

from oracle import Oracle, Oracle3D
from simplevofsolver_b200 import (DROPLET2D_ENV, DROPLETS3D_ENV, Solver, Solver3D, droplet2d, droplets3d,
                                  physical_params)

pytestmark = pytest.mark.gpu

SHAPES_2D = [  # nx, ny, uniform x (DCT along x: nx a power of two; DFT along y: ny a power of two)
    (4, 16, True), (8, 8, True), (16, 24, True), (256, 40, True), (2048, 128, True),
    (5, 4, False), (37, 8, False), (300, 64, False), (100, 1024, False), (8, 2048, False),
]
SHAPES_3D = [  # nx, ny, nz, uniform x, droplets (0: velocity only, for grids too small to hold one)
    (4, 4, 4, False, 0), (5, 16, 16, True, 0), (37, 8, 4, False, 1), (129, 4, 64, False, 1),
    (16, 256, 8, True, 1), (16, 8, 512, False, 1), (8, 2048, 4, False, 0), (8, 4, 2048, False, 0),
    (600, 8, 8, False, 1),
]


def rel(a, b, gauge, axes):
    if gauge:
        inner = tuple(slice(1, -1) for _ in range(axes))
        a = (a - a[inner].mean())[..., 1:-1]
        b = (b - b[inner].mean())[..., 1:-1]
        if axes == 2:  # the halo rows' wall cells keep the previous call's values
            a, b = a[1:-1], b[1:-1]
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("nx,ny,uniform", SHAPES_2D, ids=[f"{a}x{b}{'u' if u else 's'}" for a, b, u in SHAPES_2D])
def test_2d_shape(gpu_available, nx, ny, uniform):
    # a velocity noise of 1e-3 keeps every case's first step bounded (the
    # reference has no capillary time-step limit)
    ic = droplet2d(nx, ny, uniform=uniform, noise=1e-3)
    phys = physical_params(DROPLET2D_ENV)
    kw = dict(add_buoyancy=True, t_walls=(0.5, -0.5))
    g, o = Solver(ic, phys, **kw), Oracle(ic, phys, **kw)
    assert g.integrate() == o.run(1)[0]
    for k in ("ux", "uy", "p", "psi", "t", "vof"):
        r = rel(g.field(k), o.field(k), k in ("p", "psi"), 2)
        assert r <= 1e-12, (k, r)
    g.close()


@pytest.mark.parametrize("nx,ny,nz,uniform,ndrops", SHAPES_3D,
                         ids=[f"{a}x{b}x{c}{'u' if u else 's'}" for a, b, c, u, _ in SHAPES_3D])
def test_3d_shape(gpu_available, nx, ny, nz, uniform, ndrops):
    ic = droplets3d(nx, ny, nz, uniform=uniform, ndrops=ndrops, radii=(0.3, 0.35), seed=7)
    phys = physical_params(DROPLETS3D_ENV)
    kw = dict(add_buoyancy=True, t_walls=(0.5, -0.5))
    g, o = Solver3D(ic, phys, **kw), Oracle3D(ic, phys, **kw)
    assert g.integrate() == o.run(1)[0]
    for k in ("ux", "uy", "uz", "p", "psi", "t", "vof"):
        r = rel(g.field(k), o.field(k), k in ("p", "psi"), 3)
        assert r <= 1e-12, (k, r)
    g.close()
