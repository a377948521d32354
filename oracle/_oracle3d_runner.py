"""One replica of the 3D restatement timed on a bounded sample (TEST
INFRASTRUCTURE: the CPU baseline of bench.py).

usage: _oracle3d_runner.py N NDROPS RMIN RMAX SEED NSTEPS WARMUP OUT.npz
Builds the seeded droplet field at N^3 (simplevofsolver_b200.workloads.droplets3d),
runs WARMUP untimed and NSTEPS timed steps of oracle/svof_oracle3d.c, writes
{'seconds': ..., 'dts': ...}.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import Oracle3D  # noqa: E402
from simplevofsolver_b200.workloads import DROPLETS3D_ENV, droplets3d, physical_params  # noqa: E402


def main():
    n, nd, r0, r1, seed, steps, warm, out = sys.argv[1:9]
    ic = droplets3d(int(n), int(n), int(n), ndrops=int(nd), radii=(float(r0), float(r1)), seed=int(seed))
    o = Oracle3D(ic, physical_params(DROPLETS3D_ENV))
    o.run(int(warm))
    t0 = time.perf_counter()
    dts = o.run(int(steps))
    sec = time.perf_counter() - t0
    np.savez(out, seconds=sec, dts=dts)


if __name__ == "__main__":
    main()
