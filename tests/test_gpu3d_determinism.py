"""Repeatability of the 3D step: the same steps from the same state give the
same fields bit for bit, on the FP64 and the mixed path.

Every kernel owns its outputs (no atomics feed a result), so a difference
between two runs can only come from a race: the vof advection's cp.async
ring once waited for all but the newest copy group at the end of a plane
and so could read the next upper plane before it had landed (the mixed
path, whose FP32 fluxes are quicker, met it within ten steps at 128^3:
vof differences of 3e-50 in 15 cells, then growing).
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hashes(precision, n, steps):
    from simplevofsolver_b200.solver3d import Solver3D
    from simplevofsolver_b200.workloads import DROPLETS3D_ENV, diff3d_case, gravity3d, physical_params
    ic = diff3d_case(n)
    phys = physical_params(DROPLETS3D_ENV)
    grav, ref = gravity3d(ic)
    base = Solver3D(ic, phys)
    base.set_gravity(grav, ref)
    dts = list(base.run(steps))
    base.close()
    runs = []
    for _ in range(2):
        s = Solver3D(ic, phys, precision=precision)
        s.set_gravity(grav, ref)
        hs = []
        for dt in dts:
            s.integrate_fixed(dt)
            s.synchronize()
            h = hashlib.sha1()
            for k in ("ux", "uy", "uz", "p", "vof", "src_a", "srcuy_a"):
                h.update(np.ascontiguousarray(s.field(k)).tobytes())
            hs.append(h.hexdigest())
        runs.append(hs)
        s.close()
    return runs


@pytest.mark.parametrize("precision,steps", [("fp64", 20), ("mixed", 40)])
def test_steps_repeat_bit_for_bit(gpu_available, precision, steps):
    a, b = _hashes(precision, 128, steps)
    first = next((n for n, (x, y) in enumerate(zip(a, b)) if x != y), None)
    assert first is None, f"{precision}: the runs differ from step {first}"


@pytest.mark.parametrize("uniform", [True, False])
def test_2d_steps_repeat_bit_for_bit(gpu_available, uniform):
    """the 2D path (its line-streaming predictor keeps a per-warp cp.async
    ring; uniform x takes the DCT Poisson path, stretched x the DFT one): 30
    steps at 1024^2, twice, the same fields bit for bit"""
    from simplevofsolver_b200 import DROPLET2D_ENV, Solver, droplet2d, physical_params
    ic = droplet2d(1024, 1024, uniform=uniform)
    phys = physical_params(DROPLET2D_ENV)
    runs = []
    for _ in range(2):
        s = Solver(ic, phys)
        dts = s.run(30)
        h = hashlib.sha1(np.asarray(dts).tobytes())
        for k in ("ux", "uy", "p", "vof", "src_a", "srcuy_a"):
            h.update(np.ascontiguousarray(s.field(k)).tobytes())
        runs.append(h.hexdigest())
        s.close()
    assert runs[0] == runs[1]
