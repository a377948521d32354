"""The reference algorithm's sensitivity to one-ulp changes, measured with the
oracle (bit-identical to the reference's own sources in 2D, its 3D
restatement here).

A corner normal is the vof gradient times 1 / max(|grad vof|, DBL_EPSILON)
(src/interface/curvature_tensor.c:14-48).  In a flat cell next to the
interface the gradient is at round-off level, so a change of vof by one ulp
can turn that corner normal around; the cell's curvature then jumps by a
sizeable fraction of the largest curvature, and the CSF force on the face it
shares with an interfacial cell carries the jump into the velocity.  On a
48^3 droplet field, one ulp added to vof in one interfacial cell moves the
velocity by more than 1e-9 of its maximum after a single step, while the
same change in other cells leaves it at round-off.  This is why the CUDA
path, whose exp/log may differ from glibc's by one ulp, is compared with the
oracle function by function at full sizes (test_gpu3d_fullsize_oracle.py)
rather than along free-running trajectories.
"""
import numpy as np

from oracle import Oracle3D
from simplevofsolver_b200 import DROPLETS3D_ENV, droplets3d, physical_params


def _one_step_difference(cell_index):
    n, nd = 48, 4
    phys = physical_params(DROPLETS3D_ENV)
    ic = droplets3d(n, n, n, ndrops=nd, radii=(0.08, 0.14), seed=1)
    inter = np.argwhere((ic.vof > 0.1) & (ic.vof < 0.9))
    k, j, i = inter[cell_index * len(inter) // 8]
    ic2 = droplets3d(n, n, n, ndrops=nd, radii=(0.08, 0.14), seed=1)
    ic2.vof[k, j, i] = np.nextafter(ic2.vof[k, j, i], 2.0)
    a, b = Oracle3D(ic, phys), Oracle3D(ic2, phys)
    a.run(1)
    b.run(1)
    return max(float(np.abs(a.field(f) - b.field(f)).max() / np.abs(a.field(f)).max()) for f in ("ux", "uy", "uz"))


def test_one_ulp_in_one_cell_moves_the_velocity_by_1e_8():
    assert _one_step_difference(6) > 1e-9


def test_most_one_ulp_changes_stay_at_round_off():
    assert _one_step_difference(0) < 1e-13
