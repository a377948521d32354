"""The drop-in boundary: the reference's own host program, unchanged, on the GPU.

oracle/_ref/svof_main_ref is the reference's main.c, logging, save and
statistics code plus its solver sources, compiled here against single-rank
shims.  oracle/_ref/svof_main_dropin is the same host program with the solver
sources replaced by libsvof_b200.so's reference-signature entry points
(include/svof_reference_abi.h): fluid_init, interface_init, integrate,
fluid_save, interface_save.  Both run the same restart directory and
environment; their final restart files and logs must agree.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from simplevofsolver_b200.workloads import droplet2d, write_npy_dir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "svof_main_ref")
DROPIN_MAIN = os.path.join(ROOT, "oracle", "_ref", "svof_main_dropin")

ENV = {
    "timemax": "0.1", "wtimemax": "600", "log_rate": "0.02", "save_rate": "1e9", "save_after": "1e9",
    "stat_rate": "0.01", "stat_after": "0.04", "coef_dt_adv": "0.5", "coef_dt_dif": "0.95",
    "Ra": "1.0e4", "Pr": "1.0", "We": "10.0",
}


def run_host(exe, icdir, workdir, extra_env=None):
    for d in ("log", "save", "stat"):
        os.makedirs(os.path.join(workdir, "output", d), exist_ok=True)
    env = dict(os.environ)
    env.update(ENV)
    if extra_env:
        env.update(extra_env)
    r = subprocess.run([exe, icdir], cwd=workdir, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    saves = sorted(glob.glob(os.path.join(workdir, "output", "save", "step*")))
    assert saves, r.stdout + r.stderr
    return saves[-1], r.stdout


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference host program not built")
def test_reference_host_program_runs(tmp_path):
    """CPU: the reference program built here runs the restart directory"""
    ic = droplet2d(32, 32)
    write_npy_dir(ic, str(tmp_path / "ic"))
    last, out = run_host(REF_MAIN, str(tmp_path / "ic"), str(tmp_path / "ref"))
    assert os.path.exists(os.path.join(last, "vof.npy"))
    assert np.load(os.path.join(last, "ux.npy")).shape == (32, 33)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DROPIN_MAIN), reason="drop-in host program not built")
@pytest.mark.parametrize("uniform", [True, False])
def test_dropin_host_program_matches_reference(gpu_available, tmp_path, uniform):
    ic = droplet2d(64, 64, uniform=uniform)
    icdir = str(tmp_path / "ic")
    write_npy_dir(ic, icdir)
    ref_last, ref_out = run_host(REF_MAIN, icdir, str(tmp_path / "ref"))
    gpu_last, gpu_out = run_host(DROPIN_MAIN, icdir, str(tmp_path / "gpu"))
    assert os.path.basename(ref_last) == os.path.basename(gpu_last)  # same number of steps
    assert "B200" in gpu_out
    for k in ("ux", "uy", "t", "vof", "p"):
        a = np.load(os.path.join(gpu_last, f"{k}.npy"))
        b = np.load(os.path.join(ref_last, f"{k}.npy"))
        assert a.shape == b.shape, k
        if k == "p":  # modulo the round-off-fixed gauge constant
            a = a - a[:, 1:-1].mean()
            b = b - b[:, 1:-1].mean()
        rel = np.abs(a - b).max() / np.abs(b).max()
        assert rel <= 1e-10, (k, rel)
    for k in ("step", "time", "m_dif", "t_dif", "surface_tension", "glsizes", "lengths", "xf", "xc"):
        a = np.load(os.path.join(gpu_last, f"{k}.npy"))
        b = np.load(os.path.join(ref_last, f"{k}.npy"))
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0, err_msg=k)
    # the host's own logs, computed by the reference's logging code from the
    # fields the library leaves in managed memory
    for name in ("divergence.dat", "energy.dat", "momentum.dat", "vof.dat"):
        pa = os.path.join(str(tmp_path / "gpu"), "output", "log", name)
        pb = os.path.join(str(tmp_path / "ref"), "output", "log", name)
        if not os.path.exists(pb):
            continue
        A, B = np.loadtxt(pa, ndmin=2), np.loadtxt(pb, ndmin=2)
        assert A.shape == B.shape, name
        if name == "divergence.dat":  # max |div u| is round-off: compare magnitudes
            assert np.all(A[:, 1] < 1e-10) and np.all(B[:, 1] < 1e-10)
        else:
            np.testing.assert_allclose(A, B, rtol=1e-9, atol=1e-13, err_msg=name)
