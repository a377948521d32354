"""The two forms of the 2D predictor give identical bits.

Grids from 512 x 512 cells run the line-streaming predictor (right-hand
sides into a line array, one thread per x line for the Thomas sweeps, a
tiled update); smaller grids the fused row-tile kernel.  Both evaluate the
same expressions in the same order, so every field must be bit-identical
after several steps, whichever form a grid would pick by default
(SVOF_PREDICT_LINES forces one).  One step of the 512 x 512 droplet is also
compared with the oracle.
"""
import os

import numpy as np
import pytest

from oracle import Oracle
from simplevofsolver_b200 import DROPLET2D_ENV, Solver, droplet2d, physical_params

pytestmark = pytest.mark.gpu


def run(ic, lines, steps):
    os.environ["SVOF_PREDICT_LINES"] = "1" if lines else "0"
    try:
        s = Solver(ic, physical_params(DROPLET2D_ENV))
    finally:
        del os.environ["SVOF_PREDICT_LINES"]
    dts = s.run(steps)
    out = {k: s.field(k) for k in ("ux", "uy", "t", "p", "vof", "srcux_a", "srcuy_a", "srct_a")}
    s.close()
    return dts, out


@pytest.mark.parametrize("nx,ny,uniform", [(64, 64, True), (96, 64, False), (256, 512, True), (512, 256, False)])
def test_line_form_is_bit_identical(gpu_available, nx, ny, uniform):
    ic = droplet2d(nx, ny, uniform=uniform, noise=1e-2)
    d0, a = run(ic, False, 5)
    d1, b = run(ic, True, 5)
    assert np.array_equal(d0, d1)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_line_form_512_one_step_vs_oracle(gpu_available):
    ic = droplet2d(512, 512, noise=1e-2)
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys)  # 512 x 512: the line form by default
    o = Oracle(ic, phys)
    assert g.integrate() == o.run(1)[0]
    for k in ("ux", "uy", "vof"):
        a, b = g.field(k), o.field(k)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), k
    for k in ("p",):
        a, b = g.field(k)[1:-1], o.field(k)[1:-1]
        a = a - a[:, 1:-1].mean()
        b = b - b[:, 1:-1].mean()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), k
    g.close()
