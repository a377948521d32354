"""Restart files in the reference's layout: a solver saves its state as the
reference's save step does (step, time, the grid, the diffusivities and
surface tension, the fields' interior rows with their x ghost cells), a new
solver restarts from it, and the continued run equals the uninterrupted one.
The reference program itself reads the saved directory."""
import os
import subprocess

import numpy as np
import pytest

from simplevofsolver_b200 import (DROPLET2D_ENV, DROPLETS3D_ENV, Solver, Solver3D, droplet2d, droplets3d,
                                  physical_params)
from simplevofsolver_b200.workloads import read_npy_dir, write_npy_dir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "svof_main_ref")


def test_npy_restart_set_round_trip_3d(tmp_path):
    ic = droplets3d(16, 8, 8, ndrops=2, radii=(0.1, 0.15), seed=2)
    write_npy_dir(ic, str(tmp_path), step=7, time=0.25)
    back = read_npy_dir(str(tmp_path))
    assert (back.nx, back.ny, back.nz) == (16, 8, 8)
    for k, v in ic.fields().items():
        assert np.array_equal(v, back.fields()[k]), k
    assert np.array_equal(back.xf, ic.xf) and back.lz == ic.lz
    assert int(np.load(tmp_path / "step.npy")) == 7


@pytest.mark.gpu
@pytest.mark.parametrize("uniform", [True, False])
def test_restart_continues_bit_for_bit_2d(gpu_available, tmp_path, uniform):
    ic = droplet2d(64, 32, uniform=uniform, noise=1e-3)
    phys = physical_params(DROPLET2D_ENV)
    kw = dict(add_buoyancy=True, t_walls=(0.5, -0.5))
    whole = Solver(ic, phys, **kw)
    whole.run(6)
    first = Solver(ic, phys, **kw)
    dts = first.run(3)
    first.save(str(tmp_path / "save"), step=3, time=float(dts.sum()))
    first.close()
    again, step, time = Solver.from_npy_dir(str(tmp_path / "save"), phys, **kw)
    assert step == 3 and time == float(dts.sum())
    again.run(3)
    for k in ("ux", "uy", "p", "t", "vof"):
        assert np.array_equal(again.interior(k), whole.interior(k)), k
    saved = read_npy_dir(str(tmp_path / "save"))
    assert np.array_equal(saved.xf, ic.xf)
    assert float(np.load(tmp_path / "save" / "surface_tension.npy")) == phys["tension"]
    whole.close()
    again.close()


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference host program not built")
def test_reference_program_restarts_from_a_gpu_save(gpu_available, tmp_path):
    ic = droplet2d(32, 32, uniform=False)
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys, add_buoyancy=True, t_walls=(0.5, -0.5))
    dts = g.run(4)
    g.save(str(tmp_path / "ic"), step=4, time=float(dts.sum()))
    g.close()
    work = tmp_path / "run"
    for d in ("log", "save", "stat"):
        os.makedirs(work / "output" / d, exist_ok=True)
    env = dict(os.environ)
    env.update({"timemax": str(float(dts.sum()) + 0.02), "wtimemax": "600", "log_rate": "1e9",
                "save_rate": "1e9", "save_after": "1e9", "stat_rate": "1e9", "stat_after": "1e9",
                "coef_dt_adv": "0.5", "coef_dt_dif": "0.95", "Ra": "1.0e4", "Pr": "1.0", "We": "10.0"})
    r = subprocess.run([REF_MAIN, str(tmp_path / "ic")], cwd=str(work), env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "step: 4," in r.stdout, r.stdout


@pytest.mark.gpu
def test_restart_continues_bit_for_bit_3d(gpu_available, tmp_path):
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    whole = Solver3D(ic, phys)
    whole.run(4)
    first = Solver3D(ic, phys)
    dts = first.run(2)
    first.save(str(tmp_path / "save"), step=2, time=float(dts.sum()))
    first.close()
    again, step, time = Solver3D.from_npy_dir(str(tmp_path / "save"), phys)
    assert step == 2
    again.run(2)
    for k in ("ux", "uy", "uz", "p", "t", "vof"):
        assert np.array_equal(again.interior(k), whole.interior(k)), k
    whole.close()
    again.close()
