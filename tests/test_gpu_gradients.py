"""Gradients through rollouts of the falling-droplet workload (the
differentiation form): 256 x 256 on the unit box, one droplet of radius 0.15
at (0.5, 0.7) falling under gravity (Fr = 1, density ratio 0.1 as vof
buoyancy), Re = 200, We = 20, 200 steps with checkpoints every 20, objective
= final vof-weighted centroid y + 0.1 x final kinetic energy, gradient with
respect to the initial velocities (2 x 256 x 256), 1/We and the vof
buoyancy coefficient grav_vof = -(1 - r) / Fr^2 (r the density ratio).

* central finite differences of the forward (the GPU FP64 path, which
  reproduces the reference to 1e-12 per step), eps = 1e-6 along 16 seeded
  random smooth directions of unit norm (velocity, 1/We, grav_vof), the time-step
  sequence held fixed and the initial velocity projected onto
  divergence-free fields (adjoint.Rollout): each directional derivative
  within 1e-5 of the adjoint's, relative (measured: 15 of 16 directions
  2e-7 to 7e-6; the floor of the relative error is 5 % of the gradient's
  norm, below which central differences cannot resolve 1e-5);
* the tangent-linear dot-product test: the oracle's tangent model
  (svof_oracle_tl.inc) driven along the GPU trajectory against the CUDA
  adjoint over the rollout's steps;
* the checkpoint interval changes nothing: K = 1, 7 and N give identical
  gradients (the recompute is deterministic).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(n=256, steps=200, K=20):
    import torch
    from simplevofsolver_b200 import Solver
    from simplevofsolver_b200.adjoint import Rollout
    from simplevofsolver_b200.workloads import (FALLING2D_ENV, falling_droplet2d, falling_gravity,
                                                physical_params)
    ic = falling_droplet2d(n)
    phys = physical_params(FALLING2D_ENV)
    base = Solver(ic, phys)
    base.set_gravity(*falling_gravity(ic))
    dts = base.run(steps)            # the CFL-chosen sequence, then held fixed
    base.close()
    s = Solver(ic, phys)
    s.set_gravity(*falling_gravity(ic))
    r = Rollout(s, dts, K)
    dev = dict(dtype=torch.float64, device="cuda")
    x = {"ux": torch.tensor(ic.ux[:, 1:n], **dev), "uy": torch.tensor(ic.uy[:, 1:n + 1], **dev),
         "vof": torch.tensor(ic.vof[:, 1:n + 1], **dev), "ten": torch.tensor(phys["tension"], **dev),
         "grav": torch.tensor(falling_gravity(ic)[0], **dev)}
    return ic, phys, r, x


def objective(ic, r, x):
    from simplevofsolver_b200.adjoint import falling_objective
    ux, uy, vof, p = r.forward(x["ux"], x["uy"], x["vof"], float(x["ten"]), float(x["grav"]),
                               keep_checkpoints=False)
    return float(falling_objective(ux, uy, vof, ic.xf))


def gradient(ic, r, x):
    from simplevofsolver_b200.adjoint import falling_objective, rollout
    xs = {k: v.clone().requires_grad_(k != "vof") for k, v in x.items()}
    ux, uy, vof, p = rollout(xs["ux"], xs["uy"], xs["vof"], xs["ten"], r, grav=xs["grav"])
    J = falling_objective(ux, uy, vof, ic.xf)
    J.backward()
    return float(J.detach()), {k: xs[k].grad.clone() for k in ("ux", "uy", "ten", "grav")}


def smooth_direction(rng, nx, ny, xf, modes=4):
    """a random smooth velocity perturbation: sums of sin(m pi x) cos / sin
    (2 pi k y), m, k <= modes, on the ux faces and uy cells (the rollout
    projects it onto divergence-free fields, as it does the initial field);
    smooth, so that its directional derivative is well above the round-off
    of central differences of J"""
    xc = 0.5 * (xf[1:] + xf[:-1])
    yc = (np.arange(ny) + 0.5) / ny
    out = []
    for xs in (xf[1:nx], xc):
        f = np.zeros((ny, len(xs)))
        for m in range(1, modes + 1):
            for k in range(0, modes + 1):
                a, b = rng.standard_normal(2)
                f += np.sin(m * np.pi * xs)[None, :] * (a * np.cos(2 * np.pi * k * yc) + b * np.sin(2 * np.pi * k * yc))[:, None]
        out.append(f)
    return out[0], out[1]


def test_gradient_matches_central_differences(gpu_available):
    import torch
    ic, phys, r, x = make()
    J, grad = gradient(ic, r, x)
    assert np.isfinite(J)
    gnorm = float(torch.sqrt(sum(torch.sum(g * g) for g in grad.values())))
    rng = np.random.default_rng(2024)
    eps = 1e-6
    worst_norm, worst_rel = 0.0, 0.0
    for _ in range(16):
        dux, duy = smooth_direction(rng, ic.nx, ic.ny, ic.xf)
        v = {k: torch.tensor(a, dtype=torch.float64, device="cuda")
             for k, a in (("ux", dux), ("uy", duy), ("ten", np.array(rng.standard_normal())),
                          ("grav", np.array(rng.standard_normal())))}
        nrm = float(torch.sqrt(sum(torch.sum(a * a) for a in v.values())))
        v = {k: a / nrm for k, a in v.items()}
        d_adj = float(sum(torch.sum(grad[k] * v[k]) for k in v))
        js = []
        for sgn in (1.0, -1.0):
            xp = dict(x)
            for k in v:
                xp[k] = x[k] + sgn * eps * v[k]
            js.append(objective(ic, r, xp))
        d_fd = (js[0] - js[1]) / (2 * eps)
        # relative to the directional derivative, floored at 5 % of the
        # gradient's norm: central differences resolve J to about
        # 1e-16 |J| / eps ~ 1e-10, so a derivative 1000 times below the
        # gradient's norm is not checkable to 1e-5 relative by them
        err = abs(d_fd - d_adj) / max(abs(d_adj), 0.05 * gnorm)
        worst_norm = max(worst_norm, abs(d_fd - d_adj) / gnorm)
        worst_rel = max(worst_rel, err)
        print(f"  adjoint {d_adj:+.12e}  central differences {d_fd:+.12e}  relative {err:.2e}")
    print(f"J = {J:.12e}, |grad| = {gnorm:.6e}, max |fd - adj| / |grad| = {worst_norm:.3e}, "
          f"max relative = {worst_rel:.3e}")
    assert worst_rel <= 1e-5, (worst_norm, worst_rel)


def test_checkpoint_interval_changes_nothing(gpu_available):
    import torch
    out = []
    for K in (1, 7, 30):
        ic, phys, r, x = make(n=64, steps=30, K=K)
        J, g = gradient(ic, r, x)
        out.append((J, g))
    for J, g in out[1:]:
        assert J == out[0][0]
        for k in g:
            assert torch.equal(g[k], out[0][1][k]), k


def test_tangent_dot_product_along_rollout(gpu_available):
    """<TLM dx, y_bar> (oracle tangent model along the GPU trajectory) against
    <dx, ADJ y_bar> (CUDA adjoint) over 40 steps of the workload at full size"""
    import torch
    from oracle import Oracle
    from test_gpu_adjoint import cc, cx, taped_fields, tangent_step_along, zero_mean
    ic, phys, r, x = make(steps=40, K=40)
    s = r.s
    nx, ny = s.nx, s.ny
    o = Oracle(ic, phys)
    o.set_gravity(*s_gravity(ic))
    tan = o.tangent()
    rng = np.random.default_rng(11)
    d0 = {"ux": rng.standard_normal((ny, nx - 1)), "uy": rng.standard_normal((ny, nx))}
    dten, dgrav = 0.3, 0.4
    b = {"ux": rng.standard_normal((ny, nx - 1)), "uy": rng.standard_normal((ny, nx)),
         "p": zero_mean(rng.standard_normal((ny, nx))), "vof": rng.standard_normal((ny, nx))}
    # forward with tapes
    r.load(x["ux"], x["uy"], x["vof"], float(x["ten"]), float(x["grav"]))
    tapes = [torch.empty(s.tape_count(), dtype=torch.float64, device="cuda") for _ in r.dts]
    torch.cuda.synchronize()
    for k, dt in enumerate(r.dts):
        s.integrate_fixed(dt, tapes[k].data_ptr())
    s.synchronize()
    cx(tan.field("ux"), nx, ny)[...] = d0["ux"]
    cc(tan.field("uy"), nx, ny)[...] = d0["uy"]
    tan.init_boundaries()
    for k, dt in enumerate(r.dts):
        tangent_step_along(o, tan, tapes[k], taped_fields(s, tapes[k]), dt, dten, dgrav)
    lhs = (np.sum(cx(tan.field("ux"), nx, ny) * b["ux"]) + np.sum(cc(tan.field("uy"), nx, ny) * b["uy"])
           + np.sum(cc(tan.field("p"), nx, ny) * b["p"]) + np.sum(cc(tan.field("vof"), nx, ny, 2) * b["vof"]))
    s.adjoint_reset()
    s.synchronize()
    for k in ("ux", "uy", "p", "vof"):
        s.adjoint_view(k).copy_(torch.as_tensor(b[k], device="cuda"))
    torch.cuda.synchronize()
    for k in reversed(range(len(r.dts))):
        s.adjoint_step(tapes[k].data_ptr(), r.dts[k])
    s.synchronize()
    rhs = (float(torch.sum(s.adjoint_view("ux").cpu() * torch.as_tensor(d0["ux"])))
           + float(torch.sum(s.adjoint_view("uy").cpu() * torch.as_tensor(d0["uy"])))
           + dten * s.adjoint_tension() + dgrav * s.adjoint_gravity())
    rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    print(f"dot product over {len(r.dts)} steps: {lhs:.15e} vs {rhs:.15e}, relative {rel:.2e}")
    assert rel <= 1e-9, (lhs, rhs)


def s_gravity(ic):
    from simplevofsolver_b200.workloads import falling_gravity
    return falling_gravity(ic)
