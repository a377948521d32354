"""Queued restart-layout copies (svof3d_load_interior_async,
svof3d_store_interior_async, svof3d_io_wait): a stream of restart states
pushed through one solver with queued loads, steps and stores gives the same
fields, bit for bit, as the blocking load_interior / integrate /
store_interior sequence, and a state that comes round again gives the same
result as the first time (nothing leaks from one state into the next)."""
import numpy as np
import pytest

from simplevofsolver_b200 import DROPLETS3D_ENV, Solver3D, droplets3d, physical_params

NAMES = ["ux", "uy", "uz", "p", "t", "vof"]


def _states():
    return [droplets3d(32, 16, 16, ndrops=3, radii=(0.1, 0.2), seed=s).fields() for s in (1, 2, 3)]


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("pinned", [True, False])
def test_queued_stream_equals_blocking(gpu_available, precision, pinned):
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.1, 0.2), seed=1)
    phys = physical_params(DROPLETS3D_ENV)
    states = _states()
    order = [0, 1, 2, 0]

    blk = Solver3D(ic, phys, precision=precision)
    want = []
    for q in order:
        for k in NAMES:
            blk.load_interior(k, states[q][k])
        blk.integrate()
        want.append({k: blk.interior(k) for k in NAMES})
    blk.close()

    que = Solver3D(ic, phys, precision=precision)
    conv = _pinned if pinned else np.ascontiguousarray
    h_in = [{k: conv(v[k]) for k in NAMES} for v in states]
    got = [{k: conv(np.zeros_like(states[0][k])) for k in NAMES} for _ in order]
    for n, q in enumerate(order):
        for k in NAMES:
            que.load_interior_async(k, h_in[q][k])
        que.enqueue_steps(1)
        for k in NAMES:
            que.store_interior_async(k, got[n][k])
    que.io_wait()
    que.close()

    for n in range(len(order)):
        for k in NAMES:
            assert np.array_equal(got[n][k], want[n][k]), (n, k)
    for k in NAMES:
        assert np.array_equal(got[3][k], got[0][k]), k
    for k in ("ux", "vof"):
        assert not np.array_equal(got[1][k], got[0][k]), k


@pytest.mark.gpu
def test_queued_store_checks_its_buffer(gpu_available):
    ic = droplets3d(32, 16, 16, ndrops=3, radii=(0.1, 0.2), seed=1)
    s = Solver3D(ic, physical_params(DROPLETS3D_ENV))
    with pytest.raises(ValueError):
        s.store_interior_async("ux", np.zeros((16, 16, 34)))
    with pytest.raises(ValueError):
        s.store_interior_async("ux", np.zeros((16, 16, 33), dtype=np.float32))
    with pytest.raises(ValueError):
        s.load_interior_async("vof", np.zeros((16, 16, 33)))
    s.io_wait()
    s.close()
