"""Generates the golden fixtures of tests/test_oracle_pin.py.

Runs the reference's own sources (compiled by oracle/Makefile into
oracle/_ref/libsvof_ref*.so from the reference tree, against single-rank
shims) on small seeded droplet cases and stores the fields after 1 and 10
steps.  Needs the reference tree only to build oracle/_ref; the fixtures are
then committed so the tests can pin the oracle anywhere.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from simplevofsolver_b200.workloads import DROPLET2D_ENV, droplet2d  # noqa: E402

CASES = {
    # name: (initial condition, environment, reference build variant)
    "uniform_32x32": (lambda: droplet2d(32, 32), DROPLET2D_ENV, "c0"),
    "stretched_32x32": (lambda: droplet2d(32, 32, uniform=False), DROPLET2D_ENV, "c0"),
    "buoyant_32x16": (lambda: droplet2d(32, 16, ly=0.5, centre=(0.5, 0.25), semi_axes=(0.2, 0.1)),
                      dict(DROPLET2D_ENV, Ra=1e6, Pr=0.7), "ref"),
}
NAMES = ("ux", "uy", "p", "psi", "t", "vof")


def main():
    for name, (make, env, variant) in CASES.items():
        ic = make()
        out = {"env": np.array([env[k] for k in ("Ra", "Pr", "We", "coef_dt_adv", "coef_dt_dif")])}
        for nsteps in (1, 10):
            r = oracle.run_reference(ic, env, nsteps, variant, names=NAMES)
            out[f"dts_{nsteps}"] = r["dts"]
            for k in NAMES:
                out[f"{k}_{nsteps}"] = r[k]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
