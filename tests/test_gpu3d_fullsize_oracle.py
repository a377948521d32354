"""The 3D FP64 path against the 3D oracle at the configurations' own sizes.

Every step function of the GPU path is compared with the oracle's from the
same inputs: before each call both sides hold the oracle's fields, and the
call's outputs must agree within 1e-12 of each field's maximum (the pressure
and psi modulo their mean).  Along a trajectory this checks every function
call the step makes.

* 256^3, tanh-stretched x, 32 droplets of radii 0.04-0.08 (the FP64
  configuration's generator): the three substeps of the first step;
* 128^3, the same generator: every function call of 20 steps;
* 512^3, 128 droplets of radii 0.02-0.05 (the mixed configuration's
  generator), FP64: the three substeps of the first step.  The oracle holds
  about 40 GB of host memory here; skipped on a host with less than 96 GB.

Free-running trajectories are not compared to 1e-12 at these sizes: the
reference's algorithm itself moves the velocity by ~1e-8 in one step when
vof changes by one ulp in a single interfacial cell (corner normals of
round-off-level vof gradients, tests/test_oracle_sensitivity.py), and CUDA's
exp/log (THINC intercept and indicator) differ from glibc's by up to one
ulp.  The free-running full-size runs are checked through invariants in
test_gpu3d_fullsize.py.
"""
import numpy as np
import pytest

from oracle import Oracle3D
from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params

pytestmark = pytest.mark.gpu

TOL = 1e-12
ON = {"srcux_a": "srcux0", "srcuy_a": "srcuy0", "srcuz_a": "srcuz0", "srct_a": "srct0", "src_a": "src0",
      "srcux_b": "srcux1", "srcuy_b": "srcuy1", "srcuz_b": "srcuz1", "srct_b": "srct1", "src_b": "src1"}
STATE = ("ux", "uy", "uz", "p", "t", "vof", "psi", "srcux_a", "srcuy_a", "srcuz_a", "srct_a", "src_a",
         "srcux_b", "srcuy_b", "srcuz_b", "srct_b", "src_b")


# The THINC intercept (the normal array's fourth component) is an
# intermediate of the interface update, not a state field.  For nearly full or
# empty cells it inverts a very flat function (d intercept / d vof =
# 1 / sum_g w_g H'(z_g), up to ~1e8), so the one-ulp differences of CUDA's
# exp/log against glibc's show up there at ~1e-12 of its range; the fields
# computed from it (vof, src_a) are held to TOL.
TOL_INTERCEPT = 1e-10


def _rel(name, a, b):
    if name == "normal":
        return max(float(np.abs(a[..., :3] - b[..., :3]).max() / max(np.abs(b[..., :3]).max(), 1e-300)),
                   float(np.abs(a[..., 3] - b[..., 3]).max() / max(np.abs(b[..., 3]).max(), 1e-300)) * TOL / TOL_INTERCEPT)
    if name in ("p", "psi"):
        a = (a - a[1:-1, 1:-1, 1:-1].mean())[..., 1:-1]
        b = (b - b[1:-1, 1:-1, 1:-1].mean())[..., 1:-1]
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


class Pair:
    """the GPU solver and the oracle, compared function by function from the
    oracle's inputs"""

    def __init__(self, ic, phys):
        self.g = Solver3D(ic, phys)
        self.o = Oracle3D(ic, phys)
        self.worst = {}

    def sync_state(self, names=STATE):
        for k in names:
            self.g.set_field(k, self.o.field(ON.get(k, k)))

    def check(self, names):
        for k in names:
            r = _rel(k, self.g.field(k), self.o.field(ON.get(k, k)))
            self.worst[k] = max(self.worst.get(k, 0.0), r)
            assert r <= TOL, (k, r)

    def step(self):
        g, o = self.g, self.o
        self.sync_state()
        dt_o = o.decide_dt()
        assert g.fluid_decide_dt() == dt_o
        for rk in range(3):
            self.sync_state()
            g.interface_compute_curvature_tensor()
            o.curvature_tensor()
            self.check(["curv", "normal"])
            g.set_field("normal", o.field("normal"))
            g.set_field("curv", o.field("curv"))
            g.interface_compute_force()
            o.force()
            self.check(["ifrcx", "ifrcy", "ifrcz"])
            g.interface_update_vof(rk, dt_o)
            o.update_vof(rk, dt_o)
            self.check(["vof", "src_a"])
            self.sync_state(["vof", "src_a", "src_b"])
            g.fluid_predict_field(rk, dt_o)
            o.predict(rk, dt_o)
            self.check(["ux", "uy", "uz", "srcux_a", "srcuy_a", "srcuz_a"])
            self.sync_state(["ux", "uy", "uz", "t", "srcux_a", "srcuy_a", "srcuz_a", "srct_a", "srcux_b",
                             "srcuy_b", "srcuz_b", "srct_b"])
            g.fluid_compute_potential(rk, dt_o)
            o.potential(rk, dt_o)
            self.check(["psi"])
            self.sync_state(["psi"])
            g.fluid_correct_velocity(rk, dt_o)
            o.correct(rk, dt_o)
            self.check(["ux", "uy", "uz"])
            self.sync_state(["ux", "uy", "uz"])
            g.fluid_update_pressure(rk, dt_o)
            o.update_pressure(rk, dt_o)
            self.check(["p"])


def test_fp64_256_cubed_functions_vs_oracle(gpu_available):
    ic = droplets3d(256, 256, 256, ndrops=32, radii=(0.04, 0.08), seed=1)
    p = Pair(ic, physical_params(DROPLETS3D_ENV))
    p.step()
    print("256^3, one step, function by function:", {k: f"{v:.1e}" for k, v in p.worst.items()})
    p.g.close()


def test_fp64_128_cubed_20_steps_functions_vs_oracle(gpu_available):
    ic = droplets3d(128, 128, 128, ndrops=32, radii=(0.04, 0.08), seed=1)
    p = Pair(ic, physical_params(DROPLETS3D_ENV))
    for _ in range(20):
        p.step()
    print("128^3, 20 steps, function by function:", {k: f"{v:.1e}" for k, v in p.worst.items()})
    p.g.close()


def test_fp64_512_cubed_functions_vs_oracle(gpu_available):
    psutil = pytest.importorskip("psutil")
    if psutil.virtual_memory().available < 96e9:
        pytest.skip("the 512^3 oracle needs about 40 GB of host memory beside the solver's copies")
    ic = droplets3d(512, 512, 512, ndrops=128, radii=(0.02, 0.05), seed=1)
    p = Pair(ic, physical_params(DROPLETS3D_ENV))
    del ic
    p.step()
    print("512^3, one step, function by function:", {k: f"{v:.1e}" for k, v in p.worst.items()})
    p.g.close()
