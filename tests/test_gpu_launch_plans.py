"""Launch plans that depend on the grid.

Kernels whose shared-memory tiles hold whole lines take a dynamic
shared-memory limit that depends on the grid. That limit is an attribute of
the kernel, shared by all solvers of a process.
- A solver set up later with shorter lines must not lower the limit that an
  earlier, larger solver launches with.
- A tile of exactly 48 KB, the default limit, needs the attribute too, since
  the default also counts the kernel's static shared memory.
"""
import numpy as np
import pytest

from oracle import Oracle
from simplevofsolver_b200 import (DROPLET2D_ENV, DROPLETS3D_ENV, Solver, Solver3D, droplet2d, droplets3d,
                                  physical_params)

pytestmark = pytest.mark.gpu


def test_uniform_512_matches_oracle(gpu_available):
    # the DCT y solve of a 512-row grid stages 4 lines x 3 x 512 doubles = 48 KB
    ic = droplet2d(512, 512, uniform=True)
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys)
    o = Oracle(ic, phys)
    assert g.integrate() == o.run(1)[0]
    for k in ("ux", "uy", "vof"):
        a, b = g.field(k), o.field(k)
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), k
    g.close()


@pytest.mark.parametrize("uniform", [True, False])
def test_2d_solvers_of_different_sizes_coexist(gpu_available, uniform):
    phys = physical_params(DROPLET2D_ENV)
    big = Solver(droplet2d(1024, 256 if not uniform else 1024, uniform=uniform), phys)
    small = Solver(droplet2d(32, 32, uniform=uniform), phys)
    big.run(1)
    small.run(1)
    big.run(1)
    assert big.diagnostics()["divmax"] < 1e-8
    big.close()
    small.close()


def test_3d_solvers_of_different_sizes_coexist(gpu_available):
    phys = physical_params(DROPLETS3D_ENV)
    # the predictor coefficients stage 6 nx doubles: 96 KB at nx = 2048
    big = Solver3D(droplets3d(2048, 16, 16, ndrops=2, radii=(0.2, 0.3)), phys)
    small = Solver3D(droplets3d(16, 16, 16, ndrops=1, radii=(0.2, 0.3)), phys)
    big.run(1)
    small.run(1)
    big.run(1)
    assert big.diagnostics()["divmax"] < 1e-8
    big.close()
    small.close()
