#!/usr/bin/env python3
"""Throughput of SimpleVOFSolver's per-step hot path on B200.

A step is one call of integrate() (src/integrate.c:11-68): the CFL time step
and three Runge-Kutta substeps of interface geometry, CSF force, THINC/QQ
advection, momentum prediction with implicit-x Thomas solves, the Poisson
solve and the projection.  Metric: Mcell-steps/s = cells x steps / seconds.

Default workload: 512^3 cells, 128 seeded spherical droplets (radii 0.02 ..
0.05), tanh-stretched x grid, divergence-free random velocity (rms 0.5),
Re = 500, We = 20, FP64 (workloads.droplets3d).  The 2D workloads (the
reference's own runnable 128 x 128 droplet and larger) stay selectable.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                  [--impl ours|reference]

Our arm (default) prints one JSON line with the device-timed throughput
(inputs resident in HBM, L2 flushed between timed steps), the end-to-end
throughput through the C ABI with host buffers (restart fields copied in and
out every step), the roofline of the dominant kernel, the reference's CPU
throughput on a bounded sample, and the SM clocks seen during the timed
region.  The path does not shard (one domain per GPU): with N GPUs every rank
runs an independent replica ("weak" scaling, no collective on the data path).

The 3D line also carries the differentiation form's cost ("adjoint",
"adjoint_over_forward"): on its workload (falling droplet, 256 x 256, 200
steps, checkpoints every 20) the device time per step of the backward pass
(segment recompute with tapes plus the CUDA step adjoints) over that of the
forward (--no-adjoint skips it), the same ratio for the 3D form
("adjoint3d": the 3D differentiation workload, 256^3, 16 droplets, density
ratio 0.05, 100 steps, mixed and FP64 forwards, checkpoints fitted to a
60 GB budget), and the defect-corrected mixed form
("mixed_dc": the Poisson solve as two FP32 passes with an FP64 residual,
its throughput and its error against the FP64 path; --no-dc skips it).

--impl reference times the reference's own C implementation (its src/*.c
compiled against single-rank shims, oracle/_ref) on all host cores: one
single-rank process per core, each a replica of the same workload.  The
reference's 3D code is not part of the mounted sources, so for the 3D
workloads the CPU arms run the 3D restatement (oracle/svof_oracle3d.c) on a
bounded sample of the same generator (128^3 for the baseline line, 64^3 per
replica for the reference arm), one process per core.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Mcell-steps/s"
# the headline metric of the 3D workloads: the mixed-precision path's
# throughput at 512^3, reported beside the FP64 path's on the same GPU with
# the mixed path's error against it
METRIC3D = "Mcell-steps/s 512^3 mixed vs FP64 (same GPU, stated error)"
# 2D FP64 algorithmic HBM bytes per cell-step (103 eight-byte words: the
# compulsory reads/writes of the reference dataflow with stencil-internal
# intermediates on chip)
ALG_BYTES_CELL_STEP_2D = 824.0
# algorithmic 8-byte words per interior cell for one launch of each kernel
# kind, averaged over the three substeps (src_b is not read at substep 0)
ALG_WORDS = {
    "dt": 2.0,                 # R ux, uy
    "geom": 2.0,               # R vof, W curv (normals of interfacial cells only)
    "force": 4.0,              # R vof, curv; W ifrcx, ifrcy
    "vof": 5.0 + 2.0 / 3.0,    # R vof, ux, uy, (src_b); W vof, src_a
    "predict": 12.0 + 2.0,     # R ux uy p t ifrcx ifrcy (3 src_b); W ux uy t, 3 src_a
    "poisson_fwd": 3.0,        # R ux, uy; W spectrum
    "poisson_solve": 2.0,      # R, W spectrum
    "poisson_inv": 2.0,        # R spectrum; W psi
    "project": 7.0,            # R psi ux uy p; W ux uy p
}
KERNELS_PER_STEP = 2 + 3 * 9  # dt (2), then per substep: coef, geom, force, vof, predict, 3 Poisson, project

# 3D FP64: the ideal dataflow's compulsory 8-byte words per cell-step (145:
# per substep interface 10, momentum + scalar 20, Poisson 4 + 2 + 2 + 2 + 9,
# minus the src_b reads of substep 0, plus the CFL pass) and the words each
# kernel of this implementation moves per interior cell and launch
ALG_BYTES_CELL_STEP_3D = 1160.0
ALG_WORDS_3D = {
    "dt": 3.0,                 # R ux, uy, uz
    "geom": 2.0,               # R vof, W curv (normals of interfacial cells only)
    "force": 5.0,              # R vof, curv; W ifrcx, ifrcy, ifrcz
    "vof": 6.0 + 2.0 / 3.0,    # R vof, ux, uy, uz, (src_b); W vof, src_a
    "predict": 16.0 + 8.0 / 3.0,  # R ux uy uz p t ifrc x3 (4 src_b); W ux uy uz t, 4 src_a
    "poisson_fwd": 4.0,        # R ux, uy, uz; W half spectrum (~1 word)
    "poisson_z": 2.0,          # R, W spectrum
    "poisson_solve": 2.0,      # R, W spectrum
    "poisson_inv": 2.0,        # R spectrum; W psi
    "project": 9.0,            # R psi ux uy uz p; W ux uy uz p
}
# the mixed path's bytes per interior cell and launch: the state (velocities,
# p, t, vof, vof sources, psi) stays FP64, curvature, forces, momentum
# sources and increments are FP32; the Poisson solve is the FP64 path's
ALG_BYTES_3D_MIXED = {
    "dt": 24.0, "geom": 12.0, "force": 24.0, "vof": 48.0 + 16.0 / 3.0,
    "predict": 40.0 + 12.0 + 32.0 / 3.0 + 32.0 + 16.0,
    "poisson_fwd": 32.0, "poisson_z": 16.0, "poisson_solve": 16.0, "poisson_inv": 16.0, "project": 72.0,
}
# dt (2), then per substep: geom + intercept, force, vof, coef + rhs +
# line solve, 6 Poisson launches (right-hand side, y, z, x, z, y), project;
# the same in both paths
KERNELS_PER_STEP_3D = 2 + 3 * 14
# kernels launched per launch of a kind (profile counts kernels)
KERNELS_PER_KIND_3D = {"dt": 2, "geom": 2, "predict": 3, "poisson_fwd": 2}
KERNELS_PER_STEP_3D_MIXED = KERNELS_PER_STEP_3D

WORKLOADS3D = {
    # the headline configuration: 512^3, 128 droplets, radii 0.02 .. 0.05
    "droplets3d_512": dict(n=512, ndrops=128, radii=(0.02, 0.05)),
    # 256^3, 32 droplets, radii 0.04 .. 0.08
    "droplets3d_256": dict(n=256, ndrops=32, radii=(0.04, 0.08)),
    "droplets3d_128": dict(n=128, ndrops=32, radii=(0.04, 0.08)),
}

WORKLOADS = {
    # the reference's runnable configuration: one elliptical droplet,
    # 128 x 128, uniform x (DCT Poisson path), Re = 100, We = 10
    "droplet2d_128": dict(nx=128, ny=128, uniform=True),
    "droplet2d_1024": dict(nx=1024, ny=1024, uniform=True),
    "droplet2d_2048": dict(nx=2048, ny=2048, uniform=True),
    "droplet2d_stretched_512": dict(nx=512, ny=512, uniform=False),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region"""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return None
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference(ic, env, steps, warmup, replicas):
    import oracle
    secs = oracle.run_reference_replicas(ic, env, steps, warmup, replicas)
    return secs


def run_reference_arm_3d(args, wl, rank):
    """the 3D restatement on the host cores: one single-core replica per core
    on a 64^3 sample of the workload's generator (rank 0 only)"""
    if rank != 0:
        return
    import oracle
    ncpu = os.cpu_count() or 1
    replicas = max(1, min(ncpu, 64))
    n = 64
    try:
        secs = oracle.run_oracle3d_replicas(n, wl["ndrops"], wl["radii"], 1, args.steps, args.warmup, replicas)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"3D CPU restatement failed to run: {e}"}))
        return
    t = max(secs)
    value = replicas * n ** 3 * args.steps / t / 1e6
    sample = (f"{replicas} single-core processes x {args.steps} steps of the {args.workload} generator at "
              f"{n}^3 (3D restatement oracle/svof_oracle3d.c; the reference's 3D code is not in the mounted sources)")
    # the same metric string, unit and direction as our arm's line, so the
    # two lines compare directly; the config says what was run instead of
    # one 512^3 domain
    line = {
        "metric": METRIC3D, "value": value, "unit": METRIC, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded droplet field, workloads.droplets3d)",
        "config": {"workload": args.workload, "nx": wl["n"], "ny": wl["n"], "nz": wl["n"], "sample_n": n,
                   "replicas": replicas, "same_config": False,
                   "implementation": "restatement, not reference (oracle/svof_oracle3d.c, FP64; the reference's "
                                     "3D code is not in the mounted sources)",
                   "sample": f"{replicas} independent {n}^3 domains, one per host core"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": replicas, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_reference_arm(args, wl, ic, env, rank):
    """the reference's own C path on the host cores (rank 0 only)"""
    if rank != 0:
        return
    ncpu = os.cpu_count() or 1
    replicas = max(1, min(ncpu, 64))
    cells = wl["nx"] * wl["ny"]
    try:
        secs = cpu_reference(ic, env, args.steps, args.warmup, replicas)
    except Exception as e:  # the build of the reference is missing
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed to run: {e}"}))
        return
    t = max(secs)
    value = replicas * cells * args.steps / t / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded droplet field)",
        "config": {"workload": args.workload, "nx": wl["nx"], "ny": wl["ny"],
                   "uniform_x": wl["uniform"], "replicas": replicas},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": replicas, "kind": "reference",
                         "sample": f"{replicas} single-rank processes x {args.steps} steps of {args.workload}"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _max_over_ranks(x: float, world: int) -> float:
    """the maximum of x over the ranks (a device tensor under NCCL, a host
    tensor under gloo)"""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world: int):
    """all ranks here, and this rank's device idle"""
    import torch
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _aggregate(cells: int, steps: int, world: int, total_ms: float) -> float:
    """whole-job Mcell-steps/s of `world` replicas, each `cells` cells for
    `steps` steps, over the slowest rank's device time"""
    return world * cells * steps / (total_ms * 1e-3) / 1e6


def _timed_steps(solver, steps, world, local_rank, flush=None):
    """device time of `steps` steps enqueued back to back (events on the
    solver's stream), the max over ranks, and the clocks seen meanwhile"""
    import torch
    import torch.distributed as dist
    stream = torch.cuda.ExternalStream(solver.stream())
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for k in range(steps):
                if flush is not None:
                    flush.zero_()
                starts[k].record(stream)
                solver.enqueue_steps(1)
                ends[k].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total_ms = _max_over_ranks(float(sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))), world)
    return total_ms, clk.summary()


def adjoint_cost(steps: int = 200, K: int = 20):
    """Cost of the differentiation form on its workload (falling droplet,
    256 x 256, vof buoyancy Fr = 1, density ratio 0.1, Re = 200, We = 20):
    device time per step of the forward (svof_integrate_fixed, the time
    steps held fixed) and of the backward pass (the segment recompute with
    tapes plus the step adjoints, svof_adjoint_step), CUDA events on the
    solver's stream.  adjoint_over_forward = backward / forward per step; the
    forward's checkpoint copies are not counted on either side."""
    import torch
    from simplevofsolver_b200 import Solver
    from simplevofsolver_b200.adjoint import Rollout
    from simplevofsolver_b200.workloads import (FALLING2D_ENV, falling_droplet2d, falling_gravity,
                                                physical_params)
    n = 256
    ic = falling_droplet2d(n)
    phys = physical_params(FALLING2D_ENV)
    s = Solver(ic, phys)
    s.set_gravity(*falling_gravity(ic))
    dts = s.run(steps)
    r = Rollout(s, dts, K)
    dev = dict(dtype=torch.float64, device="cuda")
    x = (torch.tensor(ic.ux[:, 1:n], **dev), torch.tensor(ic.uy[:, 1:n + 1], **dev),
         torch.tensor(ic.vof[:, 1:n + 1], **dev), phys["tension"])
    stream = torch.cuda.ExternalStream(s.stream())
    tapes = [torch.empty(s.tape_count(), **dev) for _ in range(K)]

    def fwd():
        r.load(*x)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for dt in dts:
                s.integrate_fixed(dt)
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def bwd():
        # checkpoints of the forward (not timed), then the timed backward
        r.forward(*x)
        s.adjoint_reset()
        s.synchronize()
        ms = 0.0
        for seg in reversed(range(len(r.checkpoints))):
            n0, n1 = seg * K, min(steps, seg * K + K)
            r._restore_state(r.checkpoints[seg])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                for k in range(n0, n1):
                    s.integrate_fixed(dts[k], tapes[k - n0].data_ptr())
                for k in reversed(range(n0, n1)):
                    s.adjoint_step(tapes[k - n0].data_ptr(), dts[k])
                e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms

    fwd()
    bwd()
    f_ms = min(fwd() for _ in range(3))
    b_ms = min(bwd() for _ in range(3))
    s.close()
    return {"workload": f"falling_droplet2d_{n} (vof buoyancy Fr=1, density ratio 0.1, Re=200, We=20)",
            "steps": steps, "checkpoint_every": K, "dtype": "f64",
            "forward_ms_per_step": f_ms / steps, "backward_ms_per_step": b_ms / steps,
            "adjoint_over_forward": b_ms / f_ms,
            "backward": "segment recompute with tapes + step adjoints (svof_adjoint_step)",
            "forward": "svof_integrate_fixed (time steps held fixed)"}


def adjoint_cost3d(n: int = 256, steps: int = 100, budget: float = 60e9,
                   variants=(("mixed", "fp32"), ("mixed", "fp64"), ("fp64", "fp64"))):
    """Cost of the 3D differentiation form on its workload (diff3d_case:
    droplets3d at n^3, 16 droplets of radii in [0.05, 0.09], the vof buoyancy
    extension with density ratio 0.05 at Fr = 1, `steps` steps with the FP64
    path's CFL time-step sequence held fixed), per (forward precision,
    storage of the adjoint's intermediates) -- the adjoint's arithmetic is FP64
    in all: device time per step of the forward
    (svof3d_integrate_fixed) and of the backward pass (segment recompute with
    tapes plus svof3d_adjoint_step), CUDA events on the solver's stream;
    checkpoints every K steps, K the largest whose tapes and checkpoints fit
    `budget` bytes (adjoint.checkpoint_interval)."""
    import torch
    from simplevofsolver_b200.adjoint import Rollout3D, checkpoint_interval
    from simplevofsolver_b200.solver3d import Solver3D
    from simplevofsolver_b200.workloads import DROPLETS3D_ENV, diff3d_case, gravity3d, physical_params
    ic = diff3d_case(n)
    phys = physical_params(DROPLETS3D_ENV)
    grav, ref = gravity3d(ic)
    s = Solver3D(ic, phys)
    s.set_gravity(grav, ref)
    dts = list(s.run(steps))
    s.close()
    dev = dict(dtype=torch.float64, device="cuda")
    x = [torch.tensor(ic.ux[..., 1:n], **dev)] + [torch.tensor(getattr(ic, f)[..., 1:n + 1], **dev)
                                                  for f in ("uy", "uz", "vof")] + [phys["tension"]]
    out = {"workload": f"diff3d_{n} (droplets3d {n}^3, 16 droplets r 0.05-0.09, density ratio 0.05, Fr 1, "
                       f"{steps} steps)", "steps": steps, "hbm_budget_gb": budget / 1e9,
           "adjoint_dtype": "f64",
           "backward": "segment recompute with tapes + step adjoints (svof3d_adjoint_step)",
           "forward": "svof3d_integrate_fixed (time steps held fixed)"}
    for prec, adj in variants:
        s = Solver3D(ic, phys, precision=prec)
        s.set_gravity(grav, ref)
        s.adjoint_set_precision(adj)
        K = checkpoint_interval(s, steps, budget)
        r = Rollout3D(s, dts, K)
        stream = torch.cuda.ExternalStream(s.stream())
        tapes = [torch.empty(s.tape_count(), **dev) for _ in range(K)]

        def fwd():
            r.load(*x)
            s.synchronize()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                for dt in dts:
                    s.integrate_fixed(dt)
                e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        def bwd():
            r.forward(*x)
            s.adjoint_reset()
            s.synchronize()
            ms = 0.0
            for seg in reversed(range(len(r.checkpoints))):
                n0, n1 = seg * K, min(steps, seg * K + K)
                r._restore_state(r.checkpoints[seg])
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    e0.record(stream)
                    for k in range(n0, n1):
                        s.integrate_fixed(dts[k], tapes[k - n0].data_ptr())
                    for k in reversed(range(n0, n1)):
                        s.adjoint_step(tapes[k - n0].data_ptr(), dts[k])
                    e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
            return ms

        fwd()
        bwd()
        f_ms = min(fwd() for _ in range(2))
        b_ms = min(bwd() for _ in range(2))
        state_gb = sum(v.numel() for v in r.checkpoints[0].values()) * 8 / 1e9
        out[prec if adj == "fp64" else prec + "_adjoint_fp32"] = {
                     "forward_ms_per_step": f_ms / steps, "backward_ms_per_step": b_ms / steps,
                     "adjoint_over_forward": b_ms / f_ms, "checkpoint_every": K,
                     "tapes_gb": K * s.tape_count() * 8 / 1e9,
                     "checkpoints_gb": len(r.checkpoints) * state_gb}
        del tapes
        r.checkpoints = []
        s.close()
        torch.cuda.empty_cache()
    out["adjoint_over_forward"] = out["mixed_adjoint_fp32"]["adjoint_over_forward"]
    return out


def adjoint3d_profile_run(n: int, steps: int = 2):
    """the launches of the 3D differentiation form for a launch list: the
    differentiation workload at n^3 (FP64, vof buoyancy on), `steps` taped
    steps (svof3d_integrate_fixed) and their step adjoints
    (svof3d_adjoint_step) in reverse, seeded by the interface-area objective"""
    import torch
    from simplevofsolver_b200.adjoint import interface_area3d
    from simplevofsolver_b200.solver3d import Solver3D
    from simplevofsolver_b200.workloads import DROPLETS3D_ENV, diff3d_case, gravity3d, physical_params
    ic = diff3d_case(n)
    s = Solver3D(ic, physical_params(DROPLETS3D_ENV))
    s.set_gravity(*gravity3d(ic))
    dt = s.fluid_decide_dt()
    tapes = [torch.empty(s.tape_count(), dtype=torch.float64, device="cuda") for _ in range(steps)]
    for t in tapes:
        s.integrate_fixed(dt, t.data_ptr())
    s.synchronize()
    vof = s.device_view("vof")[2:n + 2, 2:n + 2, 1:n + 1].clone().requires_grad_(True)
    interface_area3d(vof, ic.xf, ic.ly, ic.lz).backward()
    s.adjoint_reset()
    s.synchronize()
    s.adjoint_view("vof").copy_(vof.grad)
    torch.cuda.synchronize()
    for t in reversed(tapes):
        s.adjoint_step(t.data_ptr(), dt)
    s.synchronize()
    s.close()


def _profile(solver, nprof):
    """per-kernel-kind device time of `nprof` steps launched kernel by kernel;
    a long memset ahead lets the host enqueue the whole step first"""
    import torch
    stream = torch.cuda.ExternalStream(solver.stream())
    prof = {}
    for _ in range(nprof):
        with torch.cuda.stream(stream):
            big = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
            big.zero_()
        r = solver.profile_step()
        del big
        for k, (ms, cnt) in r.items():
            acc = prof.setdefault(k, [0.0, 0])
            acc[0] += ms
            acc[1] += cnt
    return prof


def _traffic(workload, prec, kind):
    """DRAM bytes (read + write) per launch of `kind` from the committed ncu
    summary profiles/traffic.json, or None"""
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(tpath):
        return None
    with open(tpath) as f:
        tj = json.load(f)
    return tj.get(workload, {}).get(prec, {}).get(kind)


def _roofline(prof, alg_bytes_cell, cells, nprof):
    """roofline of the dominant kernel kind: algorithmic bytes per launch over
    its average device time per launch (coefficient + predictor, geometry +
    intercept and dt + final count as one launch each)"""
    dom = max(prof, key=lambda k: prof[k][0])
    nl = max(prof[dom][1] // KERNELS_PER_KIND_3D.get(dom, 1), 1)
    dom_ms = prof[dom][0] / nl
    peak, peak_kind = peaks()
    alg = alg_bytes_cell[dom] * cells
    achieved = alg / (dom_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "alg_bytes_per_launch": alg,
            "avg_launch_ms": dom_ms}


def run3d(args, wl, ic, env, world, rank, local_rank):
    """the 3D workloads: the mixed path (the headline value) and the FP64 path
    on the same GPU, the mixed path's error against the FP64 one after the
    same steps, end-to-end throughput, rooflines and the CPU baseline"""
    import torch
    import simplevofsolver_b200 as svof
    from simplevofsolver_b200.workloads import physical_params
    phys = physical_params(env)
    n = wl["n"]
    cells = n ** 3
    dxf = np.diff(ic.xf)
    vol0 = float(np.sum(ic.vof[:, :, 1:-1] * dxf)) * (ic.ly / ic.ny) * (ic.lz / ic.nz)
    res = {}
    precs = ("fp64", "mixed") if args.no_dc else ("fp64", "mixed", "mixed_dc")
    for prec in precs:
        solver = svof.Solver3D(ic, phys, precision=prec)
        solver.run(args.warmup)
        torch.cuda.synchronize()
        total_ms, clocks = _timed_steps(solver, args.steps, world, local_rank)
        diag = solver.diagnostics()
        fields = {k: solver.interior(k) for k in ("ux", "uy", "uz", "p", "vof")}
        prof = _profile(solver, 3)
        alg = ALG_BYTES_3D_MIXED if prec != "fp64" else {k: 8.0 * v for k, v in ALG_WORDS_3D.items()}
        step_alg = sum(alg[k] * (v[1] / 3) / KERNELS_PER_KIND_3D.get(k, 1) for k, v in prof.items())
        res[prec] = dict(total_ms=total_ms, clocks=clocks, diag=diag, fields=fields, prof=prof,
                         value=_aggregate(cells, args.steps, world, total_ms),
                         roofline=_roofline(prof, alg, cells, 3), step_alg_bytes=step_alg)
        if prec == "mixed":
            # end to end through the C ABI with host buffers: every step loads
            # the six restart fields from pinned host memory, takes one time
            # step and stores the six fields to a second pinned set (a stream
            # of restart states through one solver).  Queued calls: the
            # host-to-device copies of step n+1, the step n and the
            # device-to-host copies of step n-1 overlap.
            names = ["ux", "uy", "uz", "p", "t", "vof"]
            h_in = {k: torch.from_numpy(np.ascontiguousarray(ic.fields()[k])).pin_memory().numpy() for k in names}
            h_out = {k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True).numpy() for k, v in h_in.items()}
            h2d = sum(v.nbytes for v in h_in.values())

            def e2e_step():
                for nm in names:
                    solver.load_interior_async(nm, h_in[nm])
                solver.enqueue_steps(1)
                for nm in names:
                    solver.store_interior_async(nm, h_out[nm])

            e2e_step()  # makes the staging buffers and copy streams
            solver.io_wait()
            e2e_steps = max(1, args.steps)
            _barrier(world)
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                e2e_step()
            solver.io_wait()
            e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
            # the same through the blocking calls, for comparison
            store = svof.solver3d.lib3().svof3d_store_interior
            blk_steps = max(1, min(args.steps, 3))
            _barrier(world)
            t0 = time.perf_counter()
            for _ in range(blk_steps):
                for nm in names:
                    solver.load_interior(nm, h_in[nm])
                solver.integrate()
                for nm in names:
                    out = h_out[nm]
                    if store(solver._h, svof.FIELDS3D[nm], out.ctypes.data, out.size) != 0:
                        raise RuntimeError("svof3d_store_interior failed")
            blk_s = _max_over_ranks(time.perf_counter() - t0, world)
            res[prec]["e2e"] = {"value": world * cells * e2e_steps / e2e_s / 1e6, "unit": METRIC,
                                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d + 8, "steps": e2e_steps,
                                "calls": "svof3d_load_interior_async x6, svof3d_enqueue_steps(1), "
                                         "svof3d_store_interior_async x6 per step; svof3d_io_wait at the end",
                                "blocking": {"value": world * cells * blk_steps / blk_s / 1e6, "steps": blk_steps,
                                             "calls": "svof3d_load_interior x6, svof3d_integrate, "
                                                      "svof3d_store_interior x6 per step"}}
            del h_in, h_out
        solver.close()
        torch.cuda.synchronize()
    m, f = res["mixed"], res["fp64"]
    w = dxf[None, None, :]  # cell volumes up to the uniform dy * dz

    def error_vs_fp64(m):
        err = {}
        for k in ("ux", "uy", "uz", "p", "vof"):
            a, b = m["fields"][k][:, :, 1:-1], f["fields"][k][:, :, 1:-1]
            if k == "p":
                # the pressure's additive constant is fixed by round-off in
                # both paths: compare modulo the volume-weighted mean
                a = a - float(np.sum(a * w) / (np.sum(w) * a.shape[0] * a.shape[1]))
                b = b - float(np.sum(b * w) / (np.sum(w) * b.shape[0] * b.shape[1]))
            d = a - b
            err[f"{k}_rel_l2"] = float(np.linalg.norm(d.ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
            err[f"{k}_max_rel"] = float(np.abs(d).max() / max(np.abs(b).max(), 1e-300))
            del a, b, d
        err["divmax"] = m["diag"]["divmax"]
        err["volume_drift"] = abs(m["diag"]["volume"] - vol0) / vol0
        err["fp64_divmax"] = f["diag"]["divmax"]
        err["fp64_volume_drift"] = abs(f["diag"]["volume"] - vol0) / vol0
        err["after_steps"] = args.warmup + args.steps
        return err

    err = error_vs_fp64(m)
    dc = None
    if "mixed_dc" in res:
        d_ = res["mixed_dc"]
        dc = {"value": d_["value"], "unit": METRIC, "ms_per_step": d_["total_ms"] / args.steps,
              "over_fp64": d_["value"] / f["value"], "over_mixed": d_["value"] / m["value"],
              "poisson": "two FP32 passes (r2c-y, dft-z, FP32 spectrum; x line solve computing in FP64) with "
                         "the FP64 residual of the first as the second's right-hand side",
              "error": error_vs_fp64(d_),
              "kernel_ms_per_step": {k: v[0] / 3 for k, v in d_["prof"].items()}, "clocks": d_["clocks"]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            sn = 128
            ssteps = args.cpu_sample_steps or 3
            secs = oracle.run_oracle3d_replicas(sn, wl["ndrops"], wl["radii"], 1, ssteps, 1, 1)
            cpu = {"value": sn ** 3 * ssteps / secs[0] / 1e6, "unit": METRIC, "cores": 1, "kind": "port",
                   "sample": (f"{ssteps} steps of the {args.workload} generator at {sn}^3 on one core (3D "
                              "restatement oracle/svof_oracle3d.c in FP64; the reference's 3D code is not in the "
                              "mounted sources)")}
        except Exception as e:
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}

    if rank == 0:
        peak, _ = peaks()
        line = {
            "metric": METRIC3D, "value": m["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)",
            "data": "synthetic (seeded droplet field, workloads.droplets3d)",
            "config": {"workload": args.workload, "nx": n, "ny": n, "nz": n, "droplets": wl["ndrops"],
                       "radii": list(wl["radii"]), "x_grid": "tanh-stretched (1.5)",
                       "poisson": "r2c-y + dft-z + thomas-x, FP64 in both paths",
                       "precision": "mixed (FP32 interface geometry, forces, sources and increments; FP64 state, "
                                    "stencils, x line solves and Poisson solve)",
                       "l2": "not flushed: inputs larger than L2 (fields of %.1f GB resident)" % (
                           35.5 * cells * 8 / 1e9),
                       "parallelism": f"replicas{world}"},
            "fp64": {"value": f["value"], "unit": METRIC, "ms_per_step": f["total_ms"] / args.steps,
                     "roofline": dict(f["roofline"], traffic=_traffic(args.workload, "fp64", f["roofline"]["kernel"]),
                                      traffic_unit="DRAM bytes per launch (ncu, profiles/traffic.json)"),
                     "step_frac": f["value"] * 1e6 * ALG_BYTES_CELL_STEP_3D / 1e9 / peak,
                     "kernel_ms_per_step": {k: v[0] / 3 for k, v in f["prof"].items()},
                     "clocks": f["clocks"]},
            "mixed_over_fp64": m["value"] / f["value"],
            "mixed_error": err,
            "mixed_dc": dc,
            "e2e": m["e2e"],
            "gpu_launches": KERNELS_PER_STEP_3D_MIXED * args.steps,
            "roofline": dict(m["roofline"], traffic=_traffic(args.workload, "mixed", m["roofline"]["kernel"]),
                             traffic_unit="DRAM bytes per launch (ncu, profiles/traffic.json)",
                             step_frac=m["value"] * 1e6 * m["step_alg_bytes"] / 1e9 / peak,
                             step_alg_bytes_per_cell=m["step_alg_bytes"]),
            "kernel_ms_per_step": {k: v[0] / 3 for k, v in m["prof"].items()},
            "kernel_share": {k: v[0] / sum(x[0] for x in m["prof"].values()) for k, v in m["prof"].items()},
            "cpu_baseline": cpu,
            "clocks": m["clocks"],
        }
        if world == 1 and not args.no_adjoint:
            try:
                line["adjoint"] = adjoint_cost()
                line["adjoint_over_forward"] = line["adjoint"]["adjoint_over_forward"]
            except Exception as e:  # reported, never silently dropped
                line["adjoint"] = {"error": str(e)}
            try:
                line["adjoint3d"] = adjoint_cost3d()
            except Exception as e:  # reported, never silently dropped
                line["adjoint3d"] = {"error": str(e)}
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--workload", default="droplets3d_512", choices=sorted(WORKLOADS) + sorted(WORKLOADS3D))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=None)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation form's cost")
    ap.add_argument("--no-dc", action="store_true",
                    help="skip the defect-corrected mixed form (FP32 Poisson passes) in the 3D workloads")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint3d-profile", type=int, default=0, metavar="N",
                    help="profiling mode: two taped FP64 steps and their step adjoints of the 3D "
                         "differentiation workload at N^3, then exit (no JSON line)")
    args = ap.parse_args()
    if args.adjoint3d_profile:
        adjoint3d_profile_run(args.adjoint3d_profile)
        return
    three_d = args.workload in WORKLOADS3D
    if args.steps is None:
        args.steps = 20 if three_d else 200
    if args.warmup is None:
        args.warmup = 3 if three_d else 10
    args.warmup = max(args.warmup, 3)

    from simplevofsolver_b200.workloads import (DROPLET2D_ENV, DROPLETS3D_ENV, droplet2d, droplets3d,
                                                physical_params)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if three_d:
        wl = WORKLOADS3D[args.workload]
        env = DROPLETS3D_ENV
        if args.impl == "reference":
            run_reference_arm_3d(args, wl, rank)
            return
        n = wl["n"]
        ic = droplets3d(n, n, n, ndrops=wl["ndrops"], radii=wl["radii"])
        cells = n ** 3
    else:
        wl = WORKLOADS[args.workload]
        ic = droplet2d(wl["nx"], wl["ny"], uniform=wl["uniform"])
        env = DROPLET2D_ENV
        if args.impl == "reference":
            run_reference_arm(args, wl, ic, env, rank)
            return
        cells = wl["nx"] * wl["ny"]

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    import simplevofsolver_b200 as svof
    phys = physical_params(env)
    if three_d:
        run3d(args, wl, ic, env, world, rank, local_rank)
        if world > 1:
            dist.destroy_process_group()
        return
    else:
        solver = svof.Solver(ic, phys)
        names = ["ux", "uy", "p", "t", "vof"]
        lib, store, fields = svof.lib(), "svof_store_interior", svof.FIELDS
        alg_words, kernels_per_step, alg_step = ALG_WORDS, KERNELS_PER_STEP, ALG_BYTES_CELL_STEP_2D
    stream = torch.cuda.ExternalStream(solver.stream())
    # 3D: every field exceeds the 126 MB L2 many times over together; 2D:
    # flush L2 between timed steps with a 256 MB write
    flush = None if three_d else torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # warm-up (also captures the step graphs)
    solver.run(args.warmup)
    torch.cuda.synchronize()

    # ---- device-timed region: inputs resident in HBM
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                if flush is not None:
                    flush.zero_()
                starts[k].record(stream)
                solver.enqueue_steps(1)
                ends[k].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]
    total_ms = _max_over_ranks(float(sum(step_ms)), world)
    value = _aggregate(cells, args.steps, world, total_ms)
    clocks = clk.summary()

    # ---- end to end through the C ABI with host buffers: the restart fields
    # are copied in from pinned host memory and out again every step
    host = {k: torch.from_numpy(np.ascontiguousarray(ic.fields()[k])).pin_memory().numpy() for k in names}
    h2d = sum(v.nbytes for v in host.values())
    d2h = h2d + 8
    e2e_steps = max(1, min(args.steps, 3 if three_d else 50))
    store_fn = getattr(lib, store)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        for nm in names:
            solver.load_interior(nm, host[nm])
        solver.integrate()
        for nm in names:
            out = host[nm]
            rc = store_fn(solver._h, fields[nm], out.ctypes.data, out.size)
            if rc != 0:
                raise RuntimeError(f"{store} failed")
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * cells * e2e_steps / e2e_s / 1e6

    # ---- per-kernel device times (kernel by kernel, events between launches;
    # a long memset ahead lets the host enqueue the whole step first)
    prof = {}
    nprof = 3 if three_d else 5
    for _ in range(nprof):
        with torch.cuda.stream(stream):
            big = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
            big.zero_()
        r = solver.profile_step()
        del big
        for k, (ms, cnt) in r.items():
            acc = prof.setdefault(k, [0.0, 0])
            acc[0] += ms
            acc[1] += cnt
    dom = max(prof, key=lambda k: prof[k][0])
    # per launch of the dominant kind (predict: coefficient kernel + predictor
    # count as one launch of the pair)
    pair = 2 if dom in ("predict", "dt", "geom") else 1
    dom_ms = prof[dom][0] / max(prof[dom][1] // pair, 1)
    peak, peak_kind = peaks()
    alg_bytes = alg_words[dom] * 8.0 * cells
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get(args.workload, {}).get(dom)
    total_prof = sum(v[0] for v in prof.values())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if three_d:
                import oracle
                sn = 128
                ssteps = args.cpu_sample_steps or 3
                secs = oracle.run_oracle3d_replicas(sn, wl["ndrops"], wl["radii"], 1, ssteps, 1, 1)
                cpu = {"value": sn ** 3 * ssteps / secs[0] / 1e6, "unit": METRIC, "cores": 1, "kind": "port",
                       "sample": (f"{ssteps} steps of the {args.workload} generator at {sn}^3 on one core (3D "
                                  "restatement oracle/svof_oracle3d.c; the reference's 3D code is not in the "
                                  "mounted sources)")}
            else:
                ssteps = args.cpu_sample_steps or 1000
                secs = cpu_reference(ic, env, ssteps, 2, 1)
                cpu = {"value": cells * ssteps / secs[0] / 1e6, "unit": METRIC, "cores": 1, "kind": "reference",
                       "sample": f"{ssteps} steps of {args.workload}, one single-rank process"}
        except Exception as e:
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port" if three_d else "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        if three_d:
            config = {"workload": args.workload, "nx": wl["n"], "ny": wl["n"], "nz": wl["n"],
                      "droplets": wl["ndrops"], "radii": list(wl["radii"]), "x_grid": "tanh-stretched (1.5)",
                      "poisson": "r2c-y + dft-z + thomas-x", "precision": "fp64",
                      "l2": "not flushed: inputs larger than L2 (%.1f GB of fields resident)" % (
                          35.5 * cells * 8 / 1e9),
                      "parallelism": f"replicas{world}"}
        else:
            config = {"workload": args.workload, "nx": wl["nx"], "ny": wl["ny"], "uniform_x": wl["uniform"],
                      "poisson": "dct-x + periodic thomas-y" if wl["uniform"] else "r2c-y + thomas-x",
                      "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas{world}"}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": ("synthetic (seeded droplet field, workloads.droplets3d)" if three_d else
                     "synthetic (seeded droplet field, workloads.droplet2d)"),
            "config": config,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "gpu_launches": kernels_per_step * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": dom_ms,
                         "step_frac": value * 1e6 * alg_step / 1e9 / peak},
            "kernel_ms_per_step": {k: v[0] / nprof for k, v in prof.items()},
            "kernel_share": {k: v[0] / total_prof for k, v in prof.items()},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
