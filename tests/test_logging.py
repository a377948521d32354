"""Logging reductions on the device: the momentum, energy and Nusselt numbers
that the reference's logging code (src/logging/momentum.c, energy.c,
nusselt/) writes to momentum.dat, energy.dat and nusselt.dat, computed from the
GPU fields without moving them to the host (svof_logging_quantities).

The checker is the oracle's restatement of those loops (svo_logging).  It is
pinned here against the reference program itself: oracle/_ref/svof_main_ref
logs and saves at the same steps, and the restatement applied to each saved
state reproduces the logged values.  The program's logs of a 32 x 32 case
are also committed as a fixture (tests/golden/logging_32x32.npz), which the
oracle reproduces from its own trajectory where the reference cannot be
built.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import Oracle
from simplevofsolver_b200 import DROPLET2D_ENV, Solver, droplet2d, physical_params
from simplevofsolver_b200.workloads import read_npy_dir, write_npy_dir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "svof_main_ref")
# the reference's own parameters (src/param/): hot / cold walls, buoyancy
T_WALLS = (0.5, -0.5)
ENV = {
    "timemax": "0.2", "wtimemax": "600", "log_rate": "0.025", "save_rate": "0.025", "save_after": "0",
    "stat_rate": "1e9", "stat_after": "1e9", "coef_dt_adv": "0.5", "coef_dt_dif": "0.95",
    "Ra": "1.0e4", "Pr": "1.0", "We": "10.0",
}


def lively_droplet(nx, ny, uniform):
    """the 2D droplet with a temperature field and a visible velocity"""
    ic = droplet2d(nx, ny, uniform=uniform, noise=1e-2, seed=4)
    xc = ic.xc[1:-1]
    yc = (np.arange(ny) + 0.5) / ny * ic.ly
    ic.t[:, 1:-1] = 0.4 * (0.5 - xc)[None, :] + 0.1 * np.sin(2 * np.pi * yc)[:, None] * np.sin(np.pi * xc)[None, :]
    return ic


def compare(a: dict, b: dict, rtol, scale):
    for k in a:
        assert abs(a[k] - b[k]) <= rtol * max(abs(b[k]), scale[k]), (k, a[k], b[k])


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference host program not built")
def test_oracle_logging_reproduces_reference_logs(tmp_path):
    ic = lively_droplet(32, 32, uniform=False)
    icdir = str(tmp_path / "ic")
    write_npy_dir(ic, icdir)
    work = tmp_path / "run"
    for d in ("log", "save", "stat"):
        os.makedirs(work / "output" / d, exist_ok=True)
    env = dict(os.environ)
    env.update(ENV)
    r = subprocess.run([REF_MAIN, icdir], cwd=str(work), env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    logs = {name: np.loadtxt(work / "output" / "log" / f"{name}.dat", ndmin=2)
            for name in ("momentum", "energy", "nusselt")}
    nlog = logs["momentum"].shape[0]
    assert nlog >= 3
    saves = sorted(glob.glob(str(work / "output" / "save" / "step*")))
    assert len(saves) >= nlog
    phys = dict(physical_params(DROPLET2D_ENV))
    for n in range(nlog):
        st = read_npy_dir(saves[n])
        phys["m_dif"] = float(np.load(os.path.join(saves[n], "m_dif.npy")))
        phys["t_dif"] = float(np.load(os.path.join(saves[n], "t_dif.npy")))
        o = Oracle(st, phys, add_buoyancy=True, t_walls=T_WALLS)
        got = o.logging()
        ref = dict(zip(Oracle.LOGGING_NAMES, np.concatenate([logs["momentum"][n, 1:], logs["energy"][n, 1:],
                                                              logs["nusselt"][n, 1:]])))
        # the logs print 16 significant digits
        compare(got, ref, 1e-14, {k: 1e-300 for k in ref})


def test_oracle_logging_reproduces_golden():
    """the oracle runs the reference program's schedule (src/main.c:111-141,
    src/logging/main.c:25-30 and 104) and reproduces its momentum.dat,
    energy.dat and nusselt.dat, committed as a fixture by
    tests/golden/make_golden.py, to the 16 digits they print"""
    import importlib.util
    import math
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    golden = np.load(os.path.join(here, "golden", "logging_32x32.npz"))
    env = mg.LOG_ENV
    o = Oracle(mg.statistics_case(), physical_params(DROPLET2D_ENV), add_buoyancy=True, t_walls=T_WALLS)
    timemax, rate = float(env["timemax"]), float(env["log_rate"])
    time = 0.0
    nxt = rate * math.ceil(max(sys.float_info.epsilon, time) / rate)
    rows = []
    while True:
        time += o.run(1)[0]
        if timemax < time:
            break
        if nxt < time:
            rows.append(o.logging())
            nxt += rate
    assert len(rows) == golden["momentum"].shape[0] >= 5
    for n, got in enumerate(rows):
        ref = dict(zip(Oracle.LOGGING_NAMES, np.concatenate([golden["momentum"][n, 1:], golden["energy"][n, 1:],
                                                              golden["nusselt"][n, 1:]])))
        compare(got, ref, 1e-14, {k: 1e-300 for k in ref})


@pytest.mark.gpu
@pytest.mark.parametrize("uniform", [True, False])
def test_device_logging_matches_oracle(gpu_available, uniform):
    ic = lively_droplet(64, 64, uniform=uniform)
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys, add_buoyancy=True, t_walls=T_WALLS)
    o = Oracle(ic, phys, add_buoyancy=True, t_walls=T_WALLS)
    dxf, dy = np.diff(ic.xf), ic.ly / ic.ny
    for _ in range(2):
        g.run(5)
        # the same fields in both: the comparison isolates the reductions
        for k in ("ux", "uy", "t"):
            o.field(k)[...] = g.field(k)
        a, b = g.logging(), o.logging()
        # the scale of a sum whose terms cancel (momentum) is that of its terms
        scale = {k: abs(v) for k, v in b.items()}
        scale["momentum_x"] = float(np.abs(g.field("ux")[1:-1, 1:-1]).sum() * dxf.max() * dy)
        scale["momentum_y"] = float(np.abs(g.field("uy")[1:-1, 1:-1]).sum() * dxf.max() * dy)
        compare(a, b, 1e-12, scale)
    g.close()
