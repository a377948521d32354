"""Host helpers of the differentiation form (no GPU): the 3D objective and
the checkpoint interval chosen from a device-memory budget."""
import math

import numpy as np
import pytest


def test_interface_area_of_a_sphere():
    """the |grad vof| estimate of the interface area of one sphere (radius
    0.25, 64^3, uniform x) within 2 % of 4 pi r^2; a uniform field has area 0"""
    torch = pytest.importorskip("torch")
    from simplevofsolver_b200.adjoint import interface_area3d
    from simplevofsolver_b200.workloads import droplets3d
    ic = droplets3d(64, 64, 64, uniform=True, ndrops=1, radii=(0.25, 0.25), seed=2, velocity=False)
    vof = torch.tensor(ic.vof[..., 1:-1], dtype=torch.float64)
    a = float(interface_area3d(vof, ic.xf, ic.ly, ic.lz))
    assert abs(a - 4 * math.pi * 0.25 ** 2) <= 0.02 * 4 * math.pi * 0.25 ** 2, a
    assert float(interface_area3d(torch.ones_like(vof) * 0.3, ic.xf)) > 0.0  # the walls hold vof 0
    flat = torch.zeros_like(vof)
    assert float(interface_area3d(flat, ic.xf)) == 0.0
    # finite gradient where vof is uniform
    v = vof.clone().requires_grad_(True)
    interface_area3d(v, ic.xf, ic.ly, ic.lz).backward()
    assert torch.isfinite(v.grad).all()


class _FakeSolver:
    def __init__(self, n, tape):
        self.nx = self.ny = self.nz = n
        self._tape = tape

    def tape_count(self):
        return self._tape


def test_checkpoint_interval_fits_the_budget():
    from simplevofsolver_b200.adjoint import checkpoint_interval
    n = 256
    state = 8.0 * ((n + 1) * (n + 2) ** 2 + 4 * (n + 2) ** 3 + (n + 2) * (n + 4) ** 2)
    s = _FakeSolver(n, 3 * 68_800_000 + 17_600_000)
    tape = 8.0 * s.tape_count()
    for budget, steps in ((60e9, 100), (40e9, 100), (10e9, 5)):
        K = checkpoint_interval(s, steps, budget)
        assert K * tape + math.ceil(steps / K) * state <= budget
        # the next interval that is larger does not fit
        assert all(k * tape + math.ceil(steps / k) * state > budget for k in range(K + 1, steps + 1))
    assert checkpoint_interval(s, 100, 1e9) == 1   # nothing fits: one step per segment
    assert np.isclose(checkpoint_interval(s, 100, 60e9), 31)
