"""Gradients through 3D rollouts: the 3D differentiation workload at full size.

droplets3d at 256^3 (stretched x), 16 droplets of radii in [0.05, 0.09],
Re = 500, We = 20, the vof buoyancy extension with density ratio 0.05 at
Fr = 1, 100 steps with the FP64 path's CFL time-step sequence held fixed;
objective J = the interface area estimated from |grad vof| of the final vof
(adjoint.interface_area3d); gradient with respect to the initial velocity
field (3 x 256^3) and the density ratio (d grav_vof / d ratio = 1 / Fr^2).

* FP64: the adjoint's directional derivatives against central differences of
  the FP64 forward along a discretely divergence-free velocity direction
  (eps 1e-6; measured 4.5e-5, and 7.3e-4 at eps 1e-5, printed) and along the
  density ratio (eps 1e-4; measured 1.3e-4).  J carries
  about 1e-10 of noise from the forward's branches (upwind side, interfacial
  test) flipping under the perturbation, so the density-ratio derivative
  (about 1e-4) needs the larger step: measured at 100 steps, central
  differences give 2.9e-5 at eps 1e-6, 9.99e-5 at 1e-5, 9.6648e-5 at 1e-4
  and 9.6572e-5 at 1e-3, the adjoint 9.6659e-5;
* mixed (FP32 geometry, forces and sources, FP64 Poisson solve): the forward
  on the mixed path, the FP64 adjoint about its trajectory with the mixed
  paths' gradient floor (tau = 1e-5: corners whose vof varies by less than
  tau across a cell have no normal derivative; without it the transposes
  (I - n n^T) / |g| at corners of FP32-noise-sized gradients grow without
  bound over the steps); its directional derivatives along three
  divergence-free directions against the exact FP64 adjoint's, relative to
  the largest of them (measured about 5e-4, all of it the floor's: FP64 with
  the same floor differs alike), and its density-ratio derivative (measured
  1.7e-5);
* checkpoints every K steps, K the largest whose tapes and checkpoints fit a
  40 GB budget (adjoint.checkpoint_interval: K = 20 here).
The measured errors are printed (pytest -s) and bounded below.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, STEPS, BUDGET = 256, 100, 40e9


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.fixture(scope="module")
def case():
    from simplevofsolver_b200.solver3d import Solver3D
    from simplevofsolver_b200.workloads import (DROPLETS3D_ENV, diff3d_case, droplets3d, gravity3d,
                                                physical_params)
    ic = diff3d_case(N)
    phys = physical_params(DROPLETS3D_ENV)
    grav, ref = gravity3d(ic)
    s = Solver3D(ic, phys)
    s.set_gravity(grav, ref)
    dts = list(s.run(STEPS))
    s.close()
    # a discretely divergence-free velocity direction: the generator's field of another seed
    dirn = droplets3d(N, N, N, ndrops=1, radii=(0.05, 0.06), seed=7)
    return ic, phys, grav, ref, dts, dirn


def gradient(case, precision, adjoint="fp64"):
    import torch
    from simplevofsolver_b200.adjoint import Rollout3D, checkpoint_interval, interface_area3d, rollout3d
    from simplevofsolver_b200.solver3d import Solver3D
    ic, phys, grav, ref, dts, dirn = case
    s = Solver3D(ic, phys, precision=precision)
    s.set_gravity(grav, ref)
    s.adjoint_set_precision(adjoint)
    K = checkpoint_interval(s, STEPS, BUDGET)
    r = Rollout3D(s, dts, K)
    dev = dict(dtype=torch.float64, device="cuda")
    x = {"ux": torch.tensor(ic.ux[..., 1:N], **dev), "uy": torch.tensor(ic.uy[..., 1:N + 1], **dev),
         "uz": torch.tensor(ic.uz[..., 1:N + 1], **dev), "vof": torch.tensor(ic.vof[..., 1:N + 1], **dev),
         "ten": torch.tensor(phys["tension"], **dev), "grav": torch.tensor(grav, **dev)}
    xs = {k: v.clone().requires_grad_(k in ("ux", "uy", "uz", "grav")) for k, v in x.items()}
    out = rollout3d(xs["ux"], xs["uy"], xs["uz"], xs["vof"], xs["ten"], r, grav=xs["grav"])
    J = interface_area3d(out[3], ic.xf, ic.ly, ic.lz)
    J.backward()
    grads = {k: xs[k].grad.detach().clone() for k in ("ux", "uy", "uz", "grav")}
    return s, r, x, float(J.detach()), grads, K


def test_c4_gradients(case):
    import torch
    from simplevofsolver_b200.adjoint import interface_area3d
    ic, phys, grav, ref, dts, dirn = case
    dev = dict(dtype=torch.float64, device="cuda")
    d = {"ux": torch.tensor(dirn.ux[..., 1:N], **dev), "uy": torch.tensor(dirn.uy[..., 1:N + 1], **dev),
         "uz": torch.tensor(dirn.uz[..., 1:N + 1], **dev)}
    # FP64: gradient, then central differences of the FP64 forward
    s, r, x, J0, g64, K = gradient(case, "fp64")
    assert K >= 8, K

    def J(eu, er):
        with torch.no_grad():
            out = r.forward(x["ux"] + eu * d["ux"], x["uy"] + eu * d["uy"], x["uz"] + eu * d["uz"], x["vof"],
                            float(x["ten"]), grav + er, keep_checkpoints=False)
            return float(interface_area3d(out[3], ic.xf, ic.ly, ic.lz))

    fd_u = {e: (J(e, 0.0) - J(-e, 0.0)) / (2 * e) for e in (1e-6, 1e-5)}
    e = 1e-4
    fd_r = (J(0.0, e) - J(0.0, -e)) / (2 * e)
    ad_u = sum(float(torch.sum(g64[k] * d[k])) for k in d)
    ad_r = float(g64["grav"])          # d J / d ratio = d J / d grav_vof / Fr^2, Fr = 1
    print(f"\nJ = {J0:.10g}, K = {K}; velocity direction: adjoint {ad_u:.10g}, FD "
          + ", ".join(f"eps {k:.0e}: {v:.10g} (rel {rel(v, ad_u):.2e})" for k, v in fd_u.items())
          + f"; density ratio: FD {fd_r:.10g} adjoint {ad_r:.10g} rel {rel(fd_r, ad_r):.2e}")
    assert rel(fd_u[1e-6], ad_u) <= 1e-4, (fd_u, ad_u)
    assert rel(fd_r, ad_r) <= 1e-3, (fd_r, ad_r)
    r.tapes = None
    s.close()
    del r, s
    torch.cuda.empty_cache()
    # mixed forward, FP64 adjoint about its trajectory, against the FP64 adjoint
    from simplevofsolver_b200.workloads import droplets3d
    dirs = [d]
    for sd in (8, 9):
        dn = droplets3d(N, N, N, ndrops=1, radii=(0.05, 0.06), seed=sd)
        dirs.append({"ux": torch.tensor(dn.ux[..., 1:N], **dev), "uy": torch.tensor(dn.uy[..., 1:N + 1], **dev),
                     "uz": torch.tensor(dn.uz[..., 1:N + 1], **dev)})

    def directional(gk):
        return [sum(float(torch.sum(gk[k] * dd[k])) for k in dd) for dd in dirs]

    ref_dir = directional(g64)
    s, r, x, Jm, gm, Km = gradient(case, "mixed")
    mix_dir = directional(gm)
    scale = max(abs(v) for v in ref_dir)
    e_dir = max(abs(a - b) for a, b in zip(mix_dir, ref_dir)) / scale
    e_r = rel(float(gm["grav"]), float(g64["grav"]))
    print(f"mixed: J {Jm:.10g} (rel {rel(Jm, J0):.2e} to FP64); directional derivatives {mix_dir} vs FP64 "
          f"{ref_dir}: max error / max derivative {e_dir:.2e}; density-ratio derivative rel {e_r:.2e}")
    assert all(np.isfinite(mix_dir)) and np.isfinite(float(gm["grav"]))
    assert e_dir <= 2e-3 and e_r <= 1e-3, (e_dir, e_r)
    r.tapes = None
    s.close()
    del r, s
    torch.cuda.empty_cache()
    # the same with FP32 intermediates in the adjoint (the 3D differentiation
    # workload's FP32 forward and adjoint, FP64 Poisson solves)
    s, r, x, Jf, gf, Kf = gradient(case, "mixed", adjoint="fp32")
    f_dir = directional(gf)
    e_dir32 = max(abs(a - b) for a, b in zip(f_dir, ref_dir)) / scale
    e_r32 = rel(float(gf["grav"]), float(g64["grav"]))
    e_mix = max(abs(a - b) for a, b in zip(f_dir, mix_dir)) / scale
    print(f"mixed, FP32 adjoint intermediates: directional {f_dir}: max error / max derivative {e_dir32:.2e} "
          f"against the FP64 adjoint, {e_mix:.2e} against FP64 intermediates; density-ratio derivative rel "
          f"{e_r32:.2e}")
    assert all(np.isfinite(f_dir)) and np.isfinite(float(gf["grav"]))
    assert e_dir32 <= 2e-3 and e_r32 <= 1e-3 and e_mix <= 1e-4, (e_dir32, e_r32, e_mix)
    r.tapes = None
    s.close()
