"""Guard zones around every device buffer (SVOF_GUARD_BYTES): the library's
stand-in for a memory checker.

In a fresh process with 4 KB guard bands, the 2D paths (DCT and DFT Poisson
solves), the 2D adjoint step, the 3D paths (FP64, mixed, defect-corrected),
the 3D adjoint steps (FP64 and mixed), the statistics and the queued
restart copies run, and then every guard zone must be intact: no kernel
wrote outside its buffer.  As a control, a value written into the guard band
after a live buffer (memory of the same allocation, so a legal store) must
be reported.
"""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent(r'''
    import numpy as np
    import torch
    import simplevofsolver_b200 as svof
    from simplevofsolver_b200 import (DROPLET2D_ENV, DROPLETS3D_ENV, Solver, Solver3D, SvofError, droplet2d,
                                      droplets3d, physical_params, _DeviceArray)
    from simplevofsolver_b200.solver3d import storage_shape3d
    assert svof.guard_bytes() == 4096, svof.guard_bytes()
    # 2D: DCT and DFT Poisson paths, statistics, the adjoint step
    for uniform in (True, False):
        s = Solver(droplet2d(64, 64, uniform=uniform), physical_params(DROPLET2D_ENV))
        s.run(4)
        s.statistics_collect()
        tape = torch.empty(s.tape_count(), dtype=torch.float64, device="cuda")
        s.integrate_fixed(1e-3, tape.data_ptr())
        s.synchronize()
        s.adjoint_reset()
        s.adjoint_step(tape.data_ptr(), 1e-3)
        s.synchronize()
        s.close()
    # 3D: three precisions, queued restart copies, statistics; the adjoint on two of them
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.12, 0.2), seed=3)
    phys = physical_params(DROPLETS3D_ENV)
    for prec in ("fp64", "mixed", "mixed_dc"):
        g = Solver3D(ic, phys, precision=prec)
        g.run(3)
        g.statistics_collect()
        host = {k: torch.empty(v.shape, dtype=torch.float64).pin_memory().numpy() for k, v in ic.fields().items()}
        for k in host:
            g.store_interior_async(k, host[k])
        g.io_wait()
        for k in host:
            g.load_interior_async(k, host[k])
        g.enqueue_steps(1)
        g.io_wait()
        if prec != "mixed_dc":
            g.set_gravity(-0.9, 0.2)
            tapes = [torch.empty(g.tape_count(), dtype=torch.float64, device="cuda") for _ in range(2)]
            for t in tapes:
                g.integrate_fixed(1e-3, t.data_ptr())
            g.synchronize()
            g.adjoint_reset()
            for t in reversed(tapes):
                g.adjoint_step(t.data_ptr(), 1e-3)
            g.synchronize()
        if prec == "fp64":
            keep = g
        else:
            g.close()
    torch.cuda.synchronize()
    assert svof.guard_check() == 0
    # control: one value in the guard band after the live ux buffer
    ptr = keep.device_ptr("ux")
    nbytes = 8 * int(np.prod(storage_shape3d("ux", 32, 16, 16)))
    torch.as_tensor(_DeviceArray(ptr + nbytes, (1,)), device="cuda").fill_(1.0)
    torch.cuda.synchronize()
    try:
        svof.guard_check()
    except SvofError as e:
        assert "after it" in str(e), str(e)
        print("guard zones intact; the planted write reported:", e)
    else:
        raise AssertionError("the planted guard write was not reported")
''')


def test_no_kernel_writes_outside_its_buffer(gpu_available):
    env = dict(os.environ, SVOF_GUARD_BYTES="4096", PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "planted write reported" in r.stdout
