"""Time-averaged statistics on the device (svof_statistics_*, svof3d_statistics_*).

The reference collects ux, ux^2, uy, uy^2, t, t^2 and ux t into full arrays
at a fixed rate of simulation time and writes their row sums at the end of the
run (src/statistics.c; the schedule in src/main.c:137-140).

- The oracle's restatement (svo_stat_collect / svo_stat_reduce) is pinned
  here against the reference program itself, oracle/_ref/svof_main_ref. Its
  saves and its statistics fire at the same steps, so the restatement applied
  to the saved states reproduces the statistics it wrote, bit for bit. The
  program's output for a 32 x 32 case is also committed as a fixture
  (tests/golden/statistics_32x32.npz), which the oracle reproduces from its
  own trajectory where the reference cannot be built.
- The device kernels, given the same fields as the oracle, reproduce its
  sums of ux, uy, (uz,) t and ux t bit for bit. The sums of squares agree
  within 1e-13 relative: the device squares are correctly rounded products,
  and glibc's pow(x, 2.) is within one unit in the last place of them.
- The device path also runs the reference program's schedule on the GPU and
  is compared with the reference program's own output. The 2D GPU
  trajectory follows the reference within 1e-12 per step rather than bit
  for bit, and the sums of ux cancel to round-off, so this comparison is
  within 1e-10 of the summed magnitudes.
"""
import glob
import math
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import Oracle, Oracle3D
from simplevofsolver_b200 import (DROPLET2D_ENV, DROPLETS3D_ENV, STAT_NAMES, Solver, Solver3D, droplet2d,
                                  droplets3d, physical_params)
from simplevofsolver_b200.solver3d import STAT_NAMES3D
from simplevofsolver_b200.workloads import read_npy_dir, write_npy_dir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "svof_main_ref")
T_WALLS = (0.5, -0.5)  # the reference's own parameters (src/param/)
ENV = {
    "timemax": "0.12", "wtimemax": "600", "log_rate": "1e9", "save_rate": "0.01", "save_after": "0.02",
    "stat_rate": "0.01", "stat_after": "0.02", "coef_dt_adv": "0.5", "coef_dt_dif": "0.95",
    "Ra": "1.0e4", "Pr": "1.0", "We": "10.0",
}
SQUARES = ("ux2", "uy2", "uz2", "t2")


def lively_droplet(nx, ny, uniform):
    """the 2D droplet with a temperature field and a visible velocity"""
    ic = droplet2d(nx, ny, uniform=uniform, noise=1e-2, seed=4)
    xc = ic.xc[1:-1]
    yc = (np.arange(ny) + 0.5) / ny * ic.ly
    ic.t[:, 1:-1] = 0.4 * (0.5 - xc)[None, :] + 0.1 * np.sin(2 * np.pi * yc)[:, None] * np.sin(np.pi * xc)[None, :]
    return ic


def run_reference(ic, tmp_path):
    """the reference program on ic: its saved states and its statistics output"""
    icdir = str(tmp_path / "ic")
    write_npy_dir(ic, icdir)
    work = tmp_path / "run"
    for d in ("log", "save", "stat"):
        os.makedirs(work / "output" / d, exist_ok=True)
    env = dict(os.environ)
    env.update(ENV)
    r = subprocess.run([REF_MAIN, icdir], cwd=str(work), env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    stat = sorted(glob.glob(str(work / "output" / "stat" / "step*")))
    assert len(stat) == 1, stat
    ref = {k: np.load(os.path.join(stat[0], f"{k}.npy")) for k in STAT_NAMES}
    ref["num"] = int(np.load(os.path.join(stat[0], "num.npy")))
    saves = sorted(glob.glob(str(work / "output" / "save" / "step*")))
    return ref, saves


def compare(got, ref, names):
    assert got["num"] == ref["num"]
    for k in names:
        assert got[k].shape == ref[k].shape, k
        if k in SQUARES:
            np.testing.assert_allclose(got[k], ref[k], rtol=1e-13, atol=0, err_msg=k)
        else:
            assert np.array_equal(got[k], ref[k]), (k, np.abs(got[k] - ref[k]).max())


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "statistics_32x32.npz")


def test_oracle_statistics_reproduce_golden():
    """the oracle runs the reference program's schedule (src/main.c:111-141,
    src/statistics.c:59-75) and reproduces its statistics output, committed
    as a fixture by tests/golden/make_golden.py, bit for bit"""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(GOLDEN), "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    golden = np.load(GOLDEN)
    env = mg.STAT_ENV
    o = Oracle(mg.statistics_case(), physical_params(DROPLET2D_ENV), add_buoyancy=True, t_walls=T_WALLS)
    timemax, rate, after = float(env["timemax"]), float(env["stat_rate"]), float(env["stat_after"])
    time = 0.0
    nxt = rate * math.ceil(max(sys.float_info.epsilon, max(time, after)) / rate)
    while True:
        time += o.run(1)[0]
        if timemax < time:
            break
        if nxt < time:
            o.statistics_collect()
            nxt += rate
    got = o.statistics_reduced()
    assert got["num"] == int(golden["num"]) >= 4
    for k in STAT_NAMES:
        assert np.array_equal(got[k], golden[k]), (k, np.abs(got[k] - golden[k]).max())


def test_oracle3d_statistics_reduce_to_2d():
    """the 3D statistics restatement on a 2D field repeated along z: each z
    plane accumulates what the pinned 2D restatement accumulates, and the
    y-z sum is the sum of those plane sums in z order"""
    from simplevofsolver_b200.workloads import extrude_z
    ic2 = lively_droplet(32, 32, uniform=False)
    nz = 4
    phys = physical_params(DROPLET2D_ENV)
    o2 = Oracle(ic2, phys, add_buoyancy=True, t_walls=T_WALLS)
    o3 = Oracle3D(extrude_z(ic2, nz), phys, add_buoyancy=True, t_walls=T_WALLS)
    for _ in range(2):
        o2.statistics_collect()
        o3.statistics_collect()
    r2, r3 = o2.statistics_reduced(), o3.statistics_reduced()
    assert r2["num"] == r3["num"] == 2
    for k in STAT_NAMES:
        want = np.zeros_like(r2[k])
        for _ in range(nz):
            want = want + r2[k]
        assert np.array_equal(r3[k], want), k
    assert not r3["uz1"].any() and not r3["uz2"].any()


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference host program not built")
def test_oracle_statistics_reproduce_reference_output(tmp_path):
    ic = lively_droplet(32, 32, uniform=False)
    ref, saves = run_reference(ic, tmp_path)
    assert ref["num"] >= 4
    # every collection has a save at the same step; the last save is the final one
    assert len(saves) == ref["num"] + 1
    phys = physical_params(DROPLET2D_ENV)
    acc = Oracle(ic, phys, add_buoyancy=True, t_walls=T_WALLS)
    for d in saves[:ref["num"]]:
        st = Oracle(read_npy_dir(d), phys, add_buoyancy=True, t_walls=T_WALLS)
        for k in ("ux", "uy", "t"):
            acc.field(k)[...] = st.field(k)
        acc.statistics_collect()
    got = acc.statistics_reduced()
    assert got["num"] == ref["num"]
    for k in STAT_NAMES:
        assert np.array_equal(got[k], ref[k]), (k, np.abs(got[k] - ref[k]).max())


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference host program not built")
@pytest.mark.parametrize("uniform", [True, False])
def test_device_statistics_match_reference_program(gpu_available, tmp_path, uniform):
    ic = lively_droplet(64, 64, uniform=uniform)
    ref, _ = run_reference(ic, tmp_path)
    g = Solver(ic, physical_params(DROPLET2D_ENV), add_buoyancy=True, t_walls=T_WALLS)
    # src/main.c:111-141 and src/statistics.c:59-75 (the schedule)
    timemax, rate, after = float(ENV["timemax"]), float(ENV["stat_rate"]), float(ENV["stat_after"])
    time = 0.0
    nxt = rate * math.ceil(max(sys.float_info.epsilon, max(time, after)) / rate)
    while True:
        time += g.integrate()
        if timemax < time:
            break
        if nxt < time:
            g.statistics_collect()
            nxt += rate
    got = g.statistics_reduced()
    assert got["num"] == ref["num"] >= 4
    for k in STAT_NAMES:
        f = g.statistics_field(k)
        assert f.shape == (64, 65 if k in ("ux1", "ux2", "uxt") else 66)
        scale = float(np.abs(f).sum(axis=0).max())
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-10, atol=1e-10 * scale, err_msg=k)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("uniform", [True, False])
def test_device_statistics_2d_match_oracle(gpu_available, uniform):
    ic = lively_droplet(64, 64, uniform=uniform)
    phys = physical_params(DROPLET2D_ENV)
    g = Solver(ic, phys, add_buoyancy=True, t_walls=T_WALLS)
    o = Oracle(ic, phys, add_buoyancy=True, t_walls=T_WALLS)
    for _ in range(4):
        g.run(3)
        g.statistics_collect()
        # the oracle accumulates the device's own fields: the comparison isolates the statistics
        for k in ("ux", "uy", "t"):
            o.field(k)[...] = g.field(k)
        o.statistics_collect()
    compare(g.statistics_reduced(), o.statistics_reduced(), STAT_NAMES)
    g.close()


@pytest.mark.gpu
def test_device_statistics_2d_edges(gpu_available):
    import simplevofsolver_b200 as svof
    ic = lively_droplet(32, 32, uniform=True)
    g = Solver(ic, physical_params(DROPLET2D_ENV), add_buoyancy=True, t_walls=T_WALLS)
    empty = g.statistics_reduced()
    assert empty["num"] == 0 and all(not empty[k].any() for k in STAT_NAMES)
    g.statistics_collect()
    g.statistics_collect()
    two = g.statistics_reduced()
    assert two["num"] == 2
    ux = g.field("ux")[1:-1]
    np.testing.assert_allclose(two["ux1"], 2 * ux.sum(axis=0), rtol=1e-12,
                               atol=1e-12 * np.abs(ux).sum(axis=0).max())
    np.testing.assert_allclose(two["ux2"], 2 * (ux * ux).sum(axis=0), rtol=1e-12, atol=0)
    g.statistics_reset()
    again = g.statistics_reduced()
    assert again["num"] == 0 and not again["ux2"].any()
    buf = np.zeros(34)
    L = svof.lib()
    assert L.svof_statistics_reduce(g._h, 7, buf.ctypes.data, 34) != 0   # no such quantity
    assert L.svof_statistics_reduce(g._h, 0, buf.ctypes.data, 34) != 0   # ux1 has nx+1 = 33 columns
    assert L.svof_statistics_field(g._h, 2, buf.ctypes.data, 34) != 0    # uy1 holds 32 x 34 values
    with pytest.raises(ValueError):
        g.statistics_field("uz1")
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_statistics_3d_match_oracle(gpu_available, precision):
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.1, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    kw = dict(add_buoyancy=True, t_walls=T_WALLS)
    g = Solver3D(ic, phys, precision=precision, **kw)
    o = Oracle3D(ic, phys, **kw)
    for _ in range(3):
        g.run(2)
        g.statistics_collect()
        # the oracle accumulates the device's own fields: the comparison isolates the statistics
        for k in ("ux", "uy", "uz", "t"):
            o.field(k)[...] = g.field(k)
        o.statistics_collect()
    compare(g.statistics_reduced(), o.statistics_reduced(), STAT_NAMES3D)
    f = g.statistics_field("uz2")
    assert f.shape == (16, 16, 34) and (f >= 0).all()
    g.close()
