"""Generates the golden fixtures of tests/test_oracle_pin.py and
tests/test_statistics.py.

Runs the reference's own sources (compiled by oracle/Makefile into
oracle/_ref/libsvof_ref*.so from the reference tree, against single-rank
shims) on small seeded droplet cases and stores the fields after 1 and 10
steps.  The statistics and logging fixtures are outputs of the reference's
own host program (oracle/_ref/svof_main_ref: main.c, statistics.c, logging/
and the solver sources) on a 32 x 32 droplet: the row sums it writes to
output/stat with its sample count, and its momentum.dat, energy.dat and
nusselt.dat.  Needs the reference tree only to build oracle/_ref; the
fixtures are then committed so the tests can pin the oracle anywhere.

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

# the statistics case: the reference's own parameters (src/param/: buoyancy,
# hot and cold walls), samples every 0.01 from 0.02 to 0.12
STAT_ENV = {
    "timemax": "0.12", "wtimemax": "600", "log_rate": "1e9", "save_rate": "1e9", "save_after": "1e9",
    "stat_rate": "0.01", "stat_after": "0.02", "coef_dt_adv": "0.5", "coef_dt_dif": "0.95",
    "Ra": "1.0e4", "Pr": "1.0", "We": "10.0",
}
STAT_NAMES = ("ux1", "ux2", "uy1", "uy2", "t1", "t2", "uxt")


def statistics_case():
    """the 32 x 32 stretched droplet with a temperature field and a visible
    velocity"""
    ic = droplet2d(32, 32, uniform=False, noise=1e-2, seed=4)
    xc = ic.xc[1:-1]
    yc = (np.arange(ic.ny) + 0.5) / ic.ny * ic.ly
    ic.t[:, 1:-1] = 0.4 * (0.5 - xc)[None, :] + 0.1 * np.sin(2 * np.pi * yc)[:, None] * np.sin(np.pi * xc)[None, :]
    return ic


# the logging case: the same droplet, logged every 0.02 up to 0.2
LOG_ENV = dict(STAT_ENV, timemax="0.2", log_rate="0.02", stat_rate="1e9", stat_after="1e9")


def run_reference_program(env, tmp):
    """the reference's own host program on statistics_case() in tmp; returns its
    output directory"""
    import subprocess
    from simplevofsolver_b200.workloads import write_npy_dir
    exe = os.path.join(ROOT, "oracle", "_ref", "svof_main_ref")
    write_npy_dir(statistics_case(), os.path.join(tmp, "ic"))
    for d in ("log", "save", "stat"):
        os.makedirs(os.path.join(tmp, "run", "output", d))
    full = dict(os.environ)
    full.update(env)
    subprocess.run([exe, os.path.join(tmp, "ic")], cwd=os.path.join(tmp, "run"), env=full, check=True,
                   capture_output=True)
    return os.path.join(tmp, "run", "output")


def make_logging():
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        out = run_reference_program(LOG_ENV, tmp)
        logs = {name: np.loadtxt(os.path.join(out, "log", f"{name}.dat"), ndmin=2)
                for name in ("momentum", "energy", "nusselt")}
    np.savez_compressed(os.path.join(HERE, "logging_32x32.npz"), **logs)
    print("wrote logging_32x32")


def make_statistics():
    import glob
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        out = run_reference_program(STAT_ENV, tmp)
        (stat,) = glob.glob(os.path.join(out, "stat", "step*"))
        out = {k: np.load(os.path.join(stat, f"{k}.npy")) for k in STAT_NAMES}
        out["num"] = np.load(os.path.join(stat, "num.npy"))
    np.savez_compressed(os.path.join(HERE, "statistics_32x32.npz"), **out)
    print("wrote statistics_32x32")


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
    make_statistics()
    make_logging()


if __name__ == "__main__":
    main()
