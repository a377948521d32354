"""Differentiation form of the FP64 paths: gradients through a rollout
(2D: :class:`Rollout`; 3D: :class:`Rollout3D`, the same design with uz and
without the vof buoyancy extension).

``Rollout`` runs ``len(dts)`` time steps of the CUDA solver with the time-step
sequence held fixed (``svof_integrate_fixed``) and is differentiable with
respect to the initial velocities, the initial volume fraction, the
surface-tension coefficient 1/We and the coefficient grav_vof of the vof
buoyancy extension (through it the density ratio r: grav_vof =
-(1 - r) / Fr^2) through :class:`RolloutFunction`, a
``torch.autograd.Function`` whose backward pass runs the hand-written CUDA
adjoint of each step (``svof_adjoint_step``, ``csrc/k_adjoint.cu``).

Memory is bounded by recompute-from-checkpoint: the forward pass keeps the
full state every ``K`` steps only; the backward pass walks the segments in
reverse, re-runs each segment forward from its checkpoint while recording the
substep inputs of its K steps on a tape (K tapes of ``tape_count()`` doubles),
and applies the K step adjoints in reverse.  Device memory: N / K
checkpoints + K tapes.

The initial velocity is first projected onto discretely divergence-free
fields (``project_initial``, the default): the reference's curvature, taken
from normalised vof gradients, has no derivative where the gradient vanishes
(the flat bulk of a droplet), and a velocity perturbation with divergence
changes vof there; along divergence-free perturbations, the admissible ones
for an incompressible initial state, the map is differentiable, and the
projection's adjoint removes the rest from the gradient.

Tensors live on the GPU in compact layouts: ux on the interior faces
(ny, nx-1), uy, vof and p on the cells (ny, nx).  The temperature is not
differentiated (buoyancy of t must be off); the vof buoyancy extension
(``Solver.set_gravity``) is.
"""
from __future__ import annotations

import numpy as np

from . import Solver, SvofError


def _to_interior(name, a, nx, ny):
    """compact (device tensor) -> restart-file layout (numpy)"""
    a = a.detach().to("cpu").double().numpy()
    out = np.zeros((ny, nx + 1) if name == "ux" else (ny, nx + 2))
    if name == "ux":
        out[:, 1:nx] = a
    else:
        out[:, 1:nx + 1] = a
    return out


class Rollout:
    """``nsteps = len(dts)`` steps of one solver from a given initial state.

    ``solver`` is a :class:`Solver` (its p and t at construction are the
    initial p and t of every rollout); ``dts`` the fixed time steps;
    ``checkpoint_every`` = K."""

    STATE = ("ux", "uy", "p", "t", "vof")

    def __init__(self, solver: Solver, dts, checkpoint_every: int = 20, project_initial: bool = True):
        import torch
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be at least 1")
        self.s = solver
        self.dts = [float(x) for x in dts]
        self.K = int(checkpoint_every)
        self.nx, self.ny = solver.nx, solver.ny
        self.p0 = solver.interior("p")
        self.t0 = solver.interior("t")
        self.tapes = None
        self.checkpoints = []
        self.project = bool(project_initial)
        self._torch = torch

    # -- state transfer (the solver's stream and torch's are synchronised around each)
    def _sync(self):
        self.s.synchronize()
        self._torch.cuda.synchronize()

    def load(self, ux0, uy0, vof0, tension, grav=None):
        s = self.s
        s.set_tension(float(tension))
        if grav is not None:
            s.set_gravity(float(grav), s.gravity[1])
        s.load_interior("ux", _to_interior("ux", ux0, self.nx, self.ny))
        s.load_interior("uy", _to_interior("uy", uy0, self.nx, self.ny))
        s.load_interior("vof", _to_interior("vof", vof0, self.nx, self.ny))
        s.load_interior("p", self.p0)
        s.load_interior("t", self.t0)
        if self.project:
            # the discrete projection u - grad L^-1 div u of the initial
            # velocity (the Poisson solve and correction of a substep; the
            # product gamma dt cancels): a divergence-free field is kept to
            # round-off, and the gradient is the one of the admissible
            # (divergence-free) initial fields
            s.fluid_compute_potential(0, 1.0)
            s.fluid_correct_velocity(0, 1.0)

    def _save_state(self):
        self._sync()
        return {k: self.s.device_view(k).clone() for k in self.STATE}

    def _restore_state(self, st):
        self._sync()
        for k in self.STATE:
            self.s.device_view(k).copy_(st[k])
        self._torch.cuda.synchronize()

    def outputs(self):
        self._sync()
        nx, ny = self.nx, self.ny
        ux = self.s.device_view("ux")[1:ny + 1, 1:nx].clone()
        uy = self.s.device_view("uy")[1:ny + 1, 1:nx + 1].clone()
        p = self.s.device_view("p")[1:ny + 1, 1:nx + 1].clone()
        vof = self.s.device_view("vof")[2:ny + 2, 1:nx + 1].clone()
        return ux, uy, vof, p

    # -- forward: no tapes, checkpoints every K steps
    def forward(self, ux0, uy0, vof0, tension, grav=None, keep_checkpoints=True):
        self.load(ux0, uy0, vof0, tension, grav)
        self.checkpoints = []
        for n, dt in enumerate(self.dts):
            if keep_checkpoints and n % self.K == 0:
                self.checkpoints.append(self._save_state())
            self.s.integrate_fixed(dt)
        return self.outputs()

    # -- backward: recompute each segment with tapes, then its step adjoints in reverse
    def backward(self, gux, guy, gvof, gp):
        torch = self._torch
        s = self.s
        nx, ny = self.nx, self.ny
        if self.tapes is None:
            self.tapes = [torch.empty(s.tape_count(), dtype=torch.float64, device="cuda") for _ in range(self.K)]
        s.adjoint_reset()
        self._sync()
        zeros = torch.zeros
        seeds = {"ux": gux if gux is not None else zeros((ny, nx - 1), dtype=torch.float64, device="cuda"),
                 "uy": guy if guy is not None else zeros((ny, nx), dtype=torch.float64, device="cuda"),
                 "vof": gvof if gvof is not None else zeros((ny, nx), dtype=torch.float64, device="cuda"),
                 "p": gp if gp is not None else zeros((ny, nx), dtype=torch.float64, device="cuda")}
        # the pressure's additive constant is fixed by round-off: only its
        # zero-mean part has a meaningful adjoint
        seeds["p"] = seeds["p"] - seeds["p"].mean()
        for k, v in seeds.items():
            s.adjoint_view(k).copy_(v.double())
        torch.cuda.synchronize()
        N = len(self.dts)
        for seg in reversed(range(len(self.checkpoints))):
            n0 = seg * self.K
            n1 = min(N, n0 + self.K)
            self._restore_state(self.checkpoints[seg])
            for n in range(n0, n1):
                s.integrate_fixed(self.dts[n], self.tapes[n - n0].data_ptr())
            for n in reversed(range(n0, n1)):
                s.adjoint_step(self.tapes[n - n0].data_ptr(), self.dts[n])
        if self.project:
            s.adjoint_fluid_correct_velocity(0, 1.0)
            s.adjoint_fluid_compute_potential(0, 1.0)
        self._sync()
        g_ux = s.adjoint_view("ux").clone()
        g_uy = s.adjoint_view("uy").clone()
        g_vof = s.adjoint_view("vof").clone()
        g_ten = s.adjoint_tension()
        g_grav = s.adjoint_gravity()
        return g_ux, g_uy, g_vof, g_ten, g_grav


def _function():
    import torch

    class RolloutFunction(torch.autograd.Function):
        """(ux0, uy0, vof0, tension, grav) -> (ux, uy, vof, p) after the
        rollout's steps; backward through the CUDA step adjoints with
        recompute from checkpoints.  grav None keeps the solver's
        coefficient (and has no gradient)."""

        @staticmethod
        def forward(ctx, ux0, uy0, vof0, tension, grav, rollout):
            ctx.rollout = rollout
            ctx.tension_like = tension
            ctx.has_grav = grav is not None
            return rollout.forward(ux0, uy0, vof0, float(tension), None if grav is None else float(grav))

        @staticmethod
        def backward(ctx, gux, guy, gvof, gp):
            r = ctx.rollout
            g_ux, g_uy, g_vof, g_ten, g_grav = r.backward(gux, guy, gvof, gp)
            dev = ctx.tension_like.device
            gt = torch.tensor(g_ten, dtype=torch.float64, device=dev)
            gg = torch.tensor(g_grav, dtype=torch.float64, device=dev) if ctx.has_grav else None
            return g_ux, g_uy, g_vof, gt, gg, None

    return RolloutFunction


_RF = None


def rollout(ux0, uy0, vof0, tension, r: Rollout, grav=None):
    """differentiable rollout: returns (ux, uy, vof, p) after len(r.dts)
    steps; grav (a 0-d tensor, optional) sets the vof buoyancy coefficient"""
    global _RF
    if _RF is None:
        _RF = _function()
    return _RF.apply(ux0, uy0, vof0, tension, grav, r)


def _to_interior3(name, a, nx):
    """compact (device tensor, (nz, ny, nx-1 | nx)) -> restart interior (numpy)"""
    a = a.detach().to("cpu").double().numpy()
    nz, ny = a.shape[:2]
    out = np.zeros((nz, ny, nx + 1) if name == "ux" else (nz, ny, nx + 2))
    if name == "ux":
        out[..., 1:nx] = a
    else:
        out[..., 1:nx + 1] = a
    return out


class Rollout3D:
    """The 3D form of :class:`Rollout`: ``len(dts)`` steps of a
    :class:`simplevofsolver_b200.solver3d.Solver3D` (precision "fp64") with
    the time steps held fixed (``svof3d_integrate_fixed``), differentiable
    with respect to the initial ux, uy, uz, vof, 1/We and the vof buoyancy
    coefficient (``Solver3D.set_gravity``) through
    :func:`rollout3d`; the backward pass recomputes each segment of K steps
    from its checkpoint with tapes and applies the CUDA step adjoints
    (``svof3d_adjoint_step``, ``csrc/k3_adjoint.cu``) in reverse.  The
    initial velocity is projected onto discretely divergence-free fields
    first (``project_initial``), as in 2D.  Compact layouts: ux (nz, ny,
    nx-1), cells (nz, ny, nx)."""

    STATE = ("ux", "uy", "uz", "p", "t", "vof")

    def __init__(self, solver, dts, checkpoint_every: int = 20, project_initial: bool = True):
        import torch
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be at least 1")
        self.s = solver
        self.dts = [float(x) for x in dts]
        self.K = int(checkpoint_every)
        self.nx, self.ny, self.nz = solver.nx, solver.ny, solver.nz
        self.p0 = solver.interior("p")
        self.t0 = solver.interior("t")
        self.tapes = None
        self.checkpoints = []
        self.project = bool(project_initial)
        self._torch = torch

    def _sync(self):
        self.s.synchronize()
        self._torch.cuda.synchronize()

    def load(self, ux0, uy0, uz0, vof0, tension, grav=None):
        s = self.s
        s.set_tension(float(tension))
        if grav is not None:
            s.set_gravity(float(grav), s.gravity[1])
        for name, a in (("ux", ux0), ("uy", uy0), ("uz", uz0), ("vof", vof0)):
            s.load_interior(name, _to_interior3(name, a, self.nx))
        s.load_interior("p", self.p0)
        s.load_interior("t", self.t0)
        if self.project:
            s.fluid_compute_potential_dft(0, 1.0)
            s.fluid_correct_velocity(0, 1.0)

    def _save_state(self):
        self._sync()
        return {k: self.s.device_view(k).clone() for k in self.STATE}

    def _restore_state(self, st):
        self._sync()
        for k in self.STATE:
            self.s.device_view(k).copy_(st[k])
        self._torch.cuda.synchronize()

    def outputs(self):
        self._sync()
        nx, ny, nz = self.nx, self.ny, self.nz
        ux = self.s.device_view("ux")[1:nz + 1, 1:ny + 1, 1:nx].clone()
        uy = self.s.device_view("uy")[1:nz + 1, 1:ny + 1, 1:nx + 1].clone()
        uz = self.s.device_view("uz")[1:nz + 1, 1:ny + 1, 1:nx + 1].clone()
        p = self.s.device_view("p")[1:nz + 1, 1:ny + 1, 1:nx + 1].clone()
        vof = self.s.device_view("vof")[2:nz + 2, 2:ny + 2, 1:nx + 1].clone()
        return ux, uy, uz, vof, p

    def forward(self, ux0, uy0, uz0, vof0, tension, grav=None, keep_checkpoints=True):
        self.load(ux0, uy0, uz0, vof0, tension, grav)
        self.checkpoints = []
        for n, dt in enumerate(self.dts):
            if keep_checkpoints and n % self.K == 0:
                self.checkpoints.append(self._save_state())
            self.s.integrate_fixed(dt)
        return self.outputs()

    def backward(self, gux, guy, guz, gvof, gp):
        torch = self._torch
        s = self.s
        nx, ny, nz = self.nx, self.ny, self.nz
        if self.tapes is None:
            self.tapes = [torch.empty(s.tape_count(), dtype=torch.float64, device="cuda") for _ in range(self.K)]
        s.adjoint_reset()
        self._sync()
        dev = dict(dtype=torch.float64, device="cuda")
        seeds = {"ux": gux if gux is not None else torch.zeros((nz, ny, nx - 1), **dev),
                 "uy": guy if guy is not None else torch.zeros((nz, ny, nx), **dev),
                 "uz": guz if guz is not None else torch.zeros((nz, ny, nx), **dev),
                 "vof": gvof if gvof is not None else torch.zeros((nz, ny, nx), **dev),
                 "p": gp if gp is not None else torch.zeros((nz, ny, nx), **dev)}
        seeds["p"] = seeds["p"] - seeds["p"].mean()
        for k, v in seeds.items():
            s.adjoint_view(k).copy_(v.double())
        torch.cuda.synchronize()
        N = len(self.dts)
        for seg in reversed(range(len(self.checkpoints))):
            n0 = seg * self.K
            n1 = min(N, n0 + self.K)
            self._restore_state(self.checkpoints[seg])
            for n in range(n0, n1):
                s.integrate_fixed(self.dts[n], self.tapes[n - n0].data_ptr())
            for n in reversed(range(n0, n1)):
                s.adjoint_step(self.tapes[n - n0].data_ptr(), self.dts[n])
        if self.project:
            s.adjoint_fluid_correct_velocity(0, 1.0)
            s.adjoint_fluid_compute_potential_dft(0, 1.0)
        self._sync()
        return (s.adjoint_view("ux").clone(), s.adjoint_view("uy").clone(), s.adjoint_view("uz").clone(),
                s.adjoint_view("vof").clone(), s.adjoint_tension(), s.adjoint_gravity())


def _function3d():
    import torch

    class Rollout3DFunction(torch.autograd.Function):
        """(ux0, uy0, uz0, vof0, tension, grav) -> (ux, uy, uz, vof, p) after
        the rollout's steps; backward through the CUDA step adjoints.  grav
        None keeps the solver's vof buoyancy coefficient (no gradient)."""

        @staticmethod
        def forward(ctx, ux0, uy0, uz0, vof0, tension, grav, rollout):
            ctx.rollout = rollout
            ctx.tension_like = tension
            ctx.has_grav = grav is not None
            return rollout.forward(ux0, uy0, uz0, vof0, float(tension), None if grav is None else float(grav))

        @staticmethod
        def backward(ctx, gux, guy, guz, gvof, gp):
            g_ux, g_uy, g_uz, g_vof, g_ten, g_grav = ctx.rollout.backward(gux, guy, guz, gvof, gp)
            dev = ctx.tension_like.device
            gt = torch.tensor(g_ten, dtype=torch.float64, device=dev)
            gg = torch.tensor(g_grav, dtype=torch.float64, device=dev) if ctx.has_grav else None
            return g_ux, g_uy, g_uz, g_vof, gt, gg, None

    return Rollout3DFunction


_RF3 = None


def rollout3d(ux0, uy0, uz0, vof0, tension, r: Rollout3D, grav=None):
    """differentiable 3D rollout: returns (ux, uy, uz, vof, p) after
    len(r.dts) steps; grav (a 0-d tensor, optional) sets the vof buoyancy
    coefficient"""
    global _RF3
    if _RF3 is None:
        _RF3 = _function3d()
    return _RF3.apply(ux0, uy0, uz0, vof0, tension, grav, r)


def interface_area3d(vof, xf, ly: float = 1.0, lz: float = 1.0, delta: float = 1e-9):
    """the 3D differentiation workload's objective: the interface area
    estimated from |grad vof|, sum over cells of |g| dxf dy dz with g the
    cell-centred central differences of vof (x: over the centres xc(i-1),
    xc(i+1), the wall values 0 beyond the first and last cells; y, z:
    periodic) and |g| smoothed as sqrt(|g|^2 + delta^2) - delta, so that
    cells of uniform vof add exactly 0 and the gradient stays finite there.
    vof: (nz, ny, nx) tensor."""
    import torch
    nz, ny, nx = vof.shape
    dy, dz = ly / ny, lz / nz
    xf = torch.as_tensor(np.asarray(xf), dtype=torch.float64, device=vof.device)
    dxf = xf[1:] - xf[:-1]
    xc = torch.cat([xf[:1], 0.5 * (xf[1:] + xf[:-1]), xf[-1:]])           # nx + 2, walls included
    zero = torch.zeros_like(vof[..., :1])
    vx = torch.cat([zero, vof, zero], dim=-1)
    gx = (vx[..., 2:] - vx[..., :-2]) / (xc[2:] - xc[:-2])
    gy = (torch.roll(vof, -1, dims=1) - torch.roll(vof, 1, dims=1)) / (2 * dy)
    gz = (torch.roll(vof, -1, dims=0) - torch.roll(vof, 1, dims=0)) / (2 * dz)
    mag = torch.sqrt(gx * gx + gy * gy + gz * gz + delta * delta) - delta
    return torch.sum(mag * dxf[None, None, :]) * dy * dz


def checkpoint_interval(solver, nsteps: int, budget_bytes: float) -> int:
    """the largest K whose K tapes plus ceil(nsteps / K) checkpoints of the
    state (ux, uy, uz, p, t, vof) fit in budget_bytes of device memory (the
    solver's own buffers not counted); at least 1"""
    nx, ny, nz = solver.nx, solver.ny, solver.nz
    tape = 8.0 * solver.tape_count()
    state = 8.0 * ((nx + 1) * (ny + 2) * (nz + 2) + 4 * (nx + 2) * (ny + 2) * (nz + 2)
                   + (nx + 2) * (ny + 4) * (nz + 4))
    best = 1
    for K in range(1, max(1, nsteps) + 1):
        if K * tape + -(-nsteps // K) * state <= budget_bytes:
            best = K
    return best


def falling_objective(ux, uy, vof, xf, ly: float = 1.0):
    """the differentiation workload's objective: the vof-weighted centroid y
    of the droplet plus 0.1 times the kinetic energy (the reference's energy
    weights, src/logging/energy.c:41-65: ux on dxc dy, uy on dxf dy)"""
    import torch
    ny, nx = vof.shape
    dy = ly / ny
    xf = torch.as_tensor(np.asarray(xf), dtype=torch.float64, device=vof.device)
    dxf = xf[1:] - xf[:-1]
    xc = torch.cat([xf[:1], 0.5 * (xf[1:] + xf[:-1]), xf[-1:]])
    dxc = xc[1:] - xc[:-1]                              # nx + 1 face spacings
    yc = (torch.arange(ny, dtype=torch.float64, device=vof.device) + 0.5) * dy
    w = vof * dxf[None, :] * dy
    centroid = torch.sum(w * yc[:, None]) / torch.sum(w)
    ke = 0.5 * torch.sum(ux * ux * dxc[None, 1:nx] * dy) + 0.5 * torch.sum(uy * uy * dxf[None, :] * dy)
    return centroid + 0.1 * ke


__all__ = ["Rollout", "rollout", "Rollout3D", "rollout3d", "falling_objective", "interface_area3d",
           "checkpoint_interval", "SvofError"]
