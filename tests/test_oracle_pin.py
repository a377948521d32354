"""Pins the oracle (this repository's C restatement, oracle/svof_oracle.c) to
the reference itself.

* against committed golden fixtures produced by the reference's own sources
  (tests/golden/make_golden.py): bit-exact after 1 and 10 steps;
* against the reference built here from its sources (oracle/_ref), on further
  sizes and both Poisson paths, when that build is present: bit-exact.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import Oracle
from simplevofsolver_b200.workloads import DROPLET2D_ENV, droplet2d, physical_params

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

CASES = {
    "uniform_32x32": (lambda: droplet2d(32, 32), {}),
    "stretched_32x32": (lambda: droplet2d(32, 32, uniform=False), {}),
    "buoyant_32x16": (lambda: droplet2d(32, 16, ly=0.5, centre=(0.5, 0.25), semi_axes=(0.2, 0.1)),
                      dict(add_buoyancy=True, t_walls=(0.5, -0.5))),
}
NAMES = ("ux", "uy", "p", "psi", "t", "vof")


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nsteps", [1, 10])
def test_oracle_matches_golden(case, nsteps):
    g = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    Ra, Pr, We, ca, cd = g["env"]
    env = dict(Ra=Ra, Pr=Pr, We=We, coef_dt_adv=ca, coef_dt_dif=cd)
    make, kw = CASES[case]
    o = Oracle(make(), physical_params(env), **kw)
    dts = o.run(nsteps)
    assert np.array_equal(dts, g[f"dts_{nsteps}"])
    for k in NAMES:
        assert np.array_equal(o.field(k).reshape(-1), g[f"{k}_{nsteps}"].reshape(-1)), k


LIVE = {
    "uniform_64x48": lambda: droplet2d(64, 48, ly=0.75, centre=(0.5, 0.375)),
    "stretched_48x64": lambda: droplet2d(48, 64, uniform=False),
    "stretched_odd_37x40": lambda: droplet2d(37, 40, uniform=False, stretch=2.0),
}


@pytest.mark.skipif(not oracle.reference_available("c0"), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("case", list(LIVE))
def test_oracle_matches_reference_build(case):
    ic = LIVE[case]()
    r = oracle.run_reference(ic, DROPLET2D_ENV, 5, "c0", names=NAMES)
    o = Oracle(ic, physical_params(DROPLET2D_ENV))
    assert np.array_equal(o.run(5), r["dts"])
    for k in NAMES:
        assert np.array_equal(o.field(k), r[k]), k
