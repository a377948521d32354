"""simplevofsolver_b200 -- SimpleVOFSolver's per-step hot path on NVIDIA B200.

Host-side mirror of the reference's solver interface
(``include/fluid_solver.h``, ``include/interface_solver.h``,
``include/integrate.h``): the same entry-point names, argument meaning and
0 / non-zero error convention, here raising :class:`SvofError` with the
library's message.  All arithmetic runs in the CUDA library
``libsvof_b200.so`` (sm_100a) through its C ABI (``include/svof_b200.h``);
there is no CPU fallback, and importing this package on a machine where the
library is missing fails loudly.

Field storage follows the reference's in-memory layouts (x fastest, x ghost
cells and y halo rows included); ``interior`` / ``load_interior`` use the
restart-file part (rows 1..ny).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .workloads import (DROPLET2D_ENV, InitialCondition, droplet2d, physical_params,  # noqa: F401
                        read_npy_dir, write_npy_dir)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsvof_b200.so")


class SvofError(RuntimeError):
    pass


class Params(ctypes.Structure):
    """svof_params_t"""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("m_dif", ctypes.c_double), ("t_dif", ctypes.c_double),
                ("tension", ctypes.c_double),
                ("coef_dt_adv", ctypes.c_double), ("coef_dt_dif", ctypes.c_double),
                ("add_buoyancy", ctypes.c_int),
                ("uy_xm", ctypes.c_double), ("uy_xp", ctypes.c_double),
                ("t_xm", ctypes.c_double), ("t_xp", ctypes.c_double)]


FIELDS = {"ux": 0, "uy": 1, "p": 2, "psi": 3, "t": 4, "vof": 5, "curv": 6, "normal": 7,
          "ifrcx": 8, "ifrcy": 9, "srcux_a": 10, "srcux_b": 11, "srcuy_a": 12, "srcuy_b": 13,
          "srct_a": 14, "srct_b": 15, "src_a": 16, "src_b": 17}

# public C-ABI symbols (include/svof_b200.h)
EXPORTS = ["svof_create", "svof_destroy", "svof_field_count", "svof_upload_field",
           "svof_download_field", "svof_device_field", "svof_load_interior", "svof_store_interior",
           "svof_x_grid_is_uniform", "svof_fluid_decide_dt", "svof_interface_compute_curvature_tensor",
           "svof_interface_compute_force", "svof_interface_update_vof", "svof_fluid_predict_field",
           "svof_fluid_compute_potential_dct", "svof_fluid_compute_potential_dft",
           "svof_fluid_correct_velocity", "svof_fluid_update_pressure", "svof_integrate", "svof_run",
           "svof_enqueue_steps", "svof_last_dt",
           "svof_diagnostics", "svof_profile_step", "svof_synchronize", "svof_stream", "svof_last_error",
           "svof_logging_quantities", "svof_statistics_collect", "svof_statistics_reset",
           "svof_statistics_count", "svof_statistics_reduce", "svof_statistics_field",
           "svof_set_gravity", "svof_set_params", "svof_tape_count", "svof_integrate_fixed",
           "svof_adjoint_field", "svof_adjoint_reset", "svof_adjoint_step", "svof_adjoint_fluid_update_pressure",
           "svof_adjoint_fluid_correct_velocity", "svof_adjoint_fluid_compute_potential",
           "svof_adjoint_fluid_predict_field", "svof_adjoint_interface_update_vof",
           "svof_adjoint_interface_compute_force", "svof_adjoint_interface_compute_curvature_tensor",
           "svof_adjoint_tension", "svof_adjoint_gravity", "svof_poisson_dct_noalloc",
           "svof_guard_bytes", "svof_guard_check"]

# adjoint fields (SVOF_ADJ_*); compact layouts: ux faces (ny, nx-1), cells (ny, nx)
ADJ_FIELDS = {"ux": 0, "uy": 1, "p": 2, "vof": 3, "psi": 4, "ifrcx": 5, "ifrcy": 6, "curv": 7, "normal": 8,
              "srcux_a": 9, "srcuy_a": 10, "src_a": 11, "tension": 12, "gravity": 13}


def adjoint_shape(name: str, nx: int, ny: int):
    if name in ("ux", "ifrcx", "srcux_a"):
        return (ny, nx - 1)
    if name == "normal":
        return (ny, nx, 3)
    return (ny, nx)


class _DeviceArray:
    """__cuda_array_interface__ of a float64 device buffer (a zero-copy view
    for torch.as_tensor)"""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}

# statistics quantities (SVOF_STAT_*), in the reference's order (src/statistics.c:41-47)
STAT_NAMES = ["ux1", "ux2", "uy1", "uy2", "t1", "t2", "uxt"]


def storage_shape(name: str, nx: int, ny: int):
    if name == "ux":
        return (ny + 2, nx + 1)
    if name in ("uy", "p", "psi", "t", "curv"):
        return (ny + 2, nx + 2)
    if name == "vof":
        return (ny + 4, nx + 2)
    if name == "normal":
        return (ny + 2, nx, 3)
    if name in ("ifrcx", "srcux_a", "srcux_b"):
        return (ny, nx - 1)
    if name in ("ifrcy", "srcuy_a", "srcuy_b", "srct_a", "srct_b", "src_a", "src_b"):
        return (ny, nx)
    raise KeyError(name)


def interior_shape(name: str, nx: int, ny: int):
    return (ny, nx + 1) if name == "ux" else (ny, nx + 2)


_lib = None


def lib() -> ctypes.CDLL:
    """The CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SvofError(f"{LIB_PATH} is missing: build it with 'python -m simplevofsolver_b200.build'")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, sz, i = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        d = ctypes.c_double
        pd = ctypes.POINTER(ctypes.c_double)
        L.svof_create.argtypes = [ctypes.POINTER(Params), dp, dp, ctypes.POINTER(vp)]
        L.svof_destroy.argtypes = [vp]
        L.svof_field_count.argtypes = [vp, i, ctypes.POINTER(sz)]
        L.svof_upload_field.argtypes = [vp, i, dp, sz]
        L.svof_download_field.argtypes = [vp, i, dp, sz]
        L.svof_device_field.argtypes = [vp, i, ctypes.POINTER(vp)]
        L.svof_load_interior.argtypes = [vp, i, dp, sz]
        L.svof_store_interior.argtypes = [vp, i, dp, sz]
        L.svof_x_grid_is_uniform.argtypes = [vp, ctypes.POINTER(i)]
        L.svof_fluid_decide_dt.argtypes = [vp, pd]
        L.svof_interface_compute_curvature_tensor.argtypes = [vp]
        L.svof_interface_compute_force.argtypes = [vp]
        for fn in ("svof_interface_update_vof", "svof_fluid_predict_field", "svof_fluid_compute_potential_dct",
                   "svof_fluid_compute_potential_dft", "svof_fluid_correct_velocity",
                   "svof_fluid_update_pressure"):
            getattr(L, fn).argtypes = [vp, sz, d]
        L.svof_integrate.argtypes = [vp, pd]
        L.svof_run.argtypes = [vp, i, dp]
        L.svof_enqueue_steps.argtypes = [vp, i]
        L.svof_last_dt.argtypes = [vp, pd]
        L.svof_diagnostics.argtypes = [vp, pd, pd, pd, pd]
        L.svof_logging_quantities.argtypes = [vp, pd, i]
        L.svof_statistics_collect.argtypes = [vp]
        L.svof_statistics_reset.argtypes = [vp]
        L.svof_statistics_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.svof_statistics_reduce.argtypes = [vp, i, dp, sz]
        L.svof_statistics_field.argtypes = [vp, i, dp, sz]
        L.svof_poisson_dct_noalloc.argtypes = [ctypes.POINTER(Params), dp, dp, dp, dp, sz, d, vp]
        L.svof_guard_bytes.argtypes = []
        L.svof_guard_bytes.restype = sz
        L.svof_guard_check.argtypes = [ctypes.POINTER(sz)]
        L.svof_synchronize.argtypes = [vp]
        L.svof_profile_step.argtypes = [vp, dp, dp, i]
        L.svof_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.svof_last_error.restype = ctypes.c_char_p
        # differentiation form
        L.svof_set_gravity.argtypes = [vp, d, d]
        L.svof_set_params.argtypes = [vp, ctypes.POINTER(Params)]
        L.svof_tape_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.svof_integrate_fixed.argtypes = [vp, d, vp]
        L.svof_adjoint_field.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        L.svof_adjoint_reset.argtypes = [vp]
        L.svof_adjoint_step.argtypes = [vp, vp, d]
        for fn in ("svof_adjoint_fluid_update_pressure", "svof_adjoint_fluid_correct_velocity",
                   "svof_adjoint_fluid_compute_potential", "svof_adjoint_fluid_predict_field",
                   "svof_adjoint_interface_update_vof"):
            getattr(L, fn).argtypes = [vp, sz, d]
        L.svof_adjoint_interface_compute_force.argtypes = [vp]
        L.svof_adjoint_interface_compute_curvature_tensor.argtypes = [vp]
        L.svof_adjoint_tension.argtypes = [vp, pd]
        L.svof_adjoint_gravity.argtypes = [vp, pd]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise SvofError(lib().svof_last_error().decode())


def guard_bytes() -> int:
    """the guard band (bytes) around every device buffer, from SVOF_GUARD_BYTES
    at allocation time; 0 = off"""
    return int(lib().svof_guard_bytes())


def guard_check() -> int:
    """scans every live guard zone; returns 0 when intact, else raises
    SvofError naming the first changed zone"""
    bad = ctypes.c_size_t(0)
    rc = lib().svof_guard_check(ctypes.byref(bad))
    if rc != 0 and bad.value == 0:
        _check(rc)
    if bad.value:
        raise SvofError(f"{bad.value} guard bytes changed: " + lib().svof_last_error().decode())
    return 0


def _c(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Solver:
    """One 2D domain on the GPU.

    ``physical`` holds m_dif, t_dif, tension, coef_dt_adv, coef_dt_dif
    (:func:`physical_params` derives them from the reference's environment
    variables Ra, Pr, We, coef_dt_adv, coef_dt_dif).  The fields of ``ic`` are
    loaded as fluid_init / interface_init load the restart files, including
    their boundary and halo update."""

    def __init__(self, ic: InitialCondition, physical: dict, add_buoyancy: bool = False,
                 uy_walls=(0.0, 0.0), t_walls=(0.0, 0.0)):
        L = lib()
        self.nx, self.ny = int(ic.nx), int(ic.ny)
        self.params = Params(self.nx, self.ny, float(ic.lx), float(ic.ly), physical["m_dif"],
                             physical["t_dif"], physical["tension"], physical["coef_dt_adv"],
                             physical["coef_dt_dif"], int(bool(add_buoyancy)), float(uy_walls[0]),
                             float(uy_walls[1]), float(t_walls[0]), float(t_walls[1]))
        self._h = ctypes.c_void_p()
        xf, xc = _c(ic.xf), _c(ic.xc)
        self._grid = (float(ic.lx), float(ic.ly), xf.copy(), xc.copy())
        self.gravity = (0.0, 0.0)  # (grav_vof, vof_ref) of the vof buoyancy extension
        _check(L.svof_create(ctypes.byref(self.params), xf.ctypes.data, xc.ctypes.data, ctypes.byref(self._h)))
        for k, v in ic.fields().items():
            self.load_interior(k, v)

    @classmethod
    def from_npy_dir(cls, dirname: str, physical: dict, **kw):
        """restart from a directory in the reference's save layout (as
        fluid_init / interface_init read it); returns (solver, step, time)"""
        ic = read_npy_dir(dirname)
        step = int(np.load(os.path.join(dirname, "step.npy")))
        time = float(np.load(os.path.join(dirname, "time.npy")))
        return cls(ic, physical, **kw), step, time

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().svof_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ data
    def field(self, name: str) -> np.ndarray:
        """copy of a field's whole device storage, shaped (rows, cols[, 3])"""
        shape = storage_shape(name, self.nx, self.ny)
        out = np.empty(shape)
        _check(lib().svof_download_field(self._h, FIELDS[name], out.ctypes.data, out.size))
        return out

    def set_field(self, name: str, a: np.ndarray):
        a = _c(a)
        if a.shape != storage_shape(name, self.nx, self.ny):
            raise ValueError(f"{name}: expected shape {storage_shape(name, self.nx, self.ny)}, got {a.shape}")
        _check(lib().svof_upload_field(self._h, FIELDS[name], a.ctypes.data, a.size))

    def load_interior(self, name: str, a: np.ndarray):
        a = _c(a)
        if a.shape != interior_shape(name, self.nx, self.ny):
            raise ValueError(f"{name}: expected shape {interior_shape(name, self.nx, self.ny)}, got {a.shape}")
        _check(lib().svof_load_interior(self._h, FIELDS[name], a.ctypes.data, a.size))

    def interior(self, name: str) -> np.ndarray:
        out = np.empty(interior_shape(name, self.nx, self.ny))
        _check(lib().svof_store_interior(self._h, FIELDS[name], out.ctypes.data, out.size))
        return out

    def device_ptr(self, name: str) -> int:
        p = ctypes.c_void_p()
        _check(lib().svof_device_field(self._h, FIELDS[name], ctypes.byref(p)))
        return int(p.value)

    def stream(self) -> int:
        p = ctypes.c_void_p()
        _check(lib().svof_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    @property
    def x_grid_is_uniform(self) -> bool:
        u = ctypes.c_int(0)
        _check(lib().svof_x_grid_is_uniform(self._h, ctypes.byref(u)))
        return bool(u.value)

    # ------------------------------------------------------------ reference entry points
    def fluid_decide_dt(self) -> float:
        dt = ctypes.c_double(0.0)
        _check(lib().svof_fluid_decide_dt(self._h, ctypes.byref(dt)))
        return dt.value

    def interface_compute_curvature_tensor(self):
        _check(lib().svof_interface_compute_curvature_tensor(self._h))

    def interface_compute_force(self):
        _check(lib().svof_interface_compute_force(self._h))

    def interface_update_vof(self, rkstep: int, dt: float):
        _check(lib().svof_interface_update_vof(self._h, rkstep, dt))

    def fluid_predict_field(self, rkstep: int, dt: float):
        _check(lib().svof_fluid_predict_field(self._h, rkstep, dt))

    def fluid_compute_potential_dct(self, rkstep: int, dt: float):
        _check(lib().svof_fluid_compute_potential_dct(self._h, rkstep, dt))

    def fluid_compute_potential_dft(self, rkstep: int, dt: float):
        _check(lib().svof_fluid_compute_potential_dft(self._h, rkstep, dt))

    def fluid_compute_potential(self, rkstep: int, dt: float):
        """the path integrate() picks (src/integrate.c:49-57)"""
        if self.x_grid_is_uniform:
            self.fluid_compute_potential_dct(rkstep, dt)
        else:
            self.fluid_compute_potential_dft(rkstep, dt)

    def fluid_correct_velocity(self, rkstep: int, dt: float):
        _check(lib().svof_fluid_correct_velocity(self._h, rkstep, dt))

    def fluid_update_pressure(self, rkstep: int, dt: float):
        _check(lib().svof_fluid_update_pressure(self._h, rkstep, dt))

    def integrate(self) -> float:
        """one time step (src/integrate.c:11-68); returns dt"""
        dt = ctypes.c_double(0.0)
        _check(lib().svof_integrate(self._h, ctypes.byref(dt)))
        return dt.value

    def run(self, nsteps: int) -> np.ndarray:
        dts = np.zeros(max(int(nsteps), 1))
        _check(lib().svof_run(self._h, int(nsteps), dts.ctypes.data))
        return dts[:nsteps]

    def enqueue_steps(self, nsteps: int):
        """enqueue nsteps steps on the solver's stream without waiting"""
        _check(lib().svof_enqueue_steps(self._h, int(nsteps)))

    def last_dt(self) -> float:
        dt = ctypes.c_double(0.0)
        _check(lib().svof_last_dt(self._h, ctypes.byref(dt)))
        return dt.value

    def diagnostics(self) -> dict:
        """max |div u| and vof min / max / volume fraction (src/logging/divergence.c,
        src/logging/interface.c)"""
        v = [ctypes.c_double() for _ in range(4)]
        _check(lib().svof_diagnostics(self._h, *[ctypes.byref(x) for x in v]))
        return dict(divmax=v[0].value, vofmin=v[1].value, vofmax=v[2].value, vofmean=v[3].value)

    # ------------------------------------------------------------ restart files
    def state(self) -> InitialCondition:
        """the current fields in the restart layout, with the grid"""
        lx, ly, xf, xc = self._grid
        return InitialCondition(self.nx, self.ny, lx, ly, xf.copy(), xc.copy(),
                                *(self.interior(k) for k in ("ux", "uy", "p", "t", "vof")))

    def fluid_save(self, dirname: str):
        """src/fluid/save.c: m_dif, t_dif and ux, uy, p, t"""
        os.makedirs(dirname, exist_ok=True)
        np.save(os.path.join(dirname, "m_dif.npy"), np.array(self.params.m_dif))
        np.save(os.path.join(dirname, "t_dif.npy"), np.array(self.params.t_dif))
        for k in ("ux", "uy", "p", "t"):
            np.save(os.path.join(dirname, f"{k}.npy"), self.interior(k))

    def interface_save(self, dirname: str):
        """src/interface/save.c: surface_tension and vof"""
        os.makedirs(dirname, exist_ok=True)
        np.save(os.path.join(dirname, "surface_tension.npy"), np.array(self.params.tension))
        np.save(os.path.join(dirname, "vof.npy"), self.interior("vof"))

    def save(self, dirname: str, step: int = 0, time: float = 0.0):
        """a save / restart directory as the reference's save entry point
        writes it (src/save.c, src/main.c:64-71, src/domain.c:60-74)"""
        write_npy_dir(self.state(), dirname, step, time)
        self.fluid_save(dirname)
        self.interface_save(dirname)

    LOGGING_NAMES = ["momentum_x", "momentum_y", "energy_ux", "energy_uy", "energy_t", "nu_heat_flux",
                     "nu_kinetic_injection", "nu_kinetic_dissipation", "nu_thermal_dissipation"]

    def logging(self) -> dict:
        """the logging reductions of src/logging/momentum.c, energy.c and
        nusselt/ on the device (the quantities of momentum.dat, energy.dat and
        nusselt.dat)"""
        out = np.zeros(9)
        _check(lib().svof_logging_quantities(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 9))
        return dict(zip(self.LOGGING_NAMES, out.tolist()))

    # ------------------------------------------------- time-averaged statistics
    def statistics_collect(self):
        """add one sample of the current fields to the device accumulators
        (src/statistics.c:117-204); queued, does not wait"""
        _check(lib().svof_statistics_collect(self._h))

    def statistics_reset(self):
        _check(lib().svof_statistics_reset(self._h))

    def statistics_count(self) -> int:
        n = ctypes.c_size_t(0)
        _check(lib().svof_statistics_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def statistics_reduced(self) -> dict:
        """the row sums reduce_and_write writes (src/statistics.c:232-281), one
        vector per quantity, plus 'num' the number of samples"""
        out = {}
        for q, k in enumerate(STAT_NAMES):
            v = np.zeros(self.nx + (1 if k in ("ux1", "ux2", "uxt") else 2))
            _check(lib().svof_statistics_reduce(self._h, q, v.ctypes.data, v.size))
            out[k] = v
        out["num"] = self.statistics_count()
        return out

    def statistics_field(self, name: str) -> np.ndarray:
        """the accumulated array of one quantity, ny x (nx+1) or ny x (nx+2)"""
        q = STAT_NAMES.index(name)
        v = np.zeros((self.ny, self.nx + (1 if name in ("ux1", "ux2", "uxt") else 2)))
        _check(lib().svof_statistics_field(self._h, q, v.ctypes.data, v.size))
        return v

    KERNEL_KINDS = ["dt", "geom", "force", "vof", "predict", "poisson_fwd", "poisson_solve",
                    "poisson_inv", "project"]

    def profile_step(self) -> dict:
        """one step launched kernel by kernel with CUDA events; {kind: (ms, launches)}"""
        n = len(self.KERNEL_KINDS)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int32)
        _check(lib().svof_profile_step(self._h, ms.ctypes.data, cnt.ctypes.data, n))
        return {k: (float(ms[q]), int(cnt[q])) for q, k in enumerate(self.KERNEL_KINDS)}

    def synchronize(self):
        _check(lib().svof_synchronize(self._h))

    # ------------------------------------------------------------ differentiation form
    def device_view(self, name: str):
        """zero-copy torch view of a field's current device storage (valid
        until the next call that swaps its buffers; synchronise the solver's
        stream and torch's around its use)"""
        import torch
        return torch.as_tensor(_DeviceArray(self.device_ptr(name), storage_shape(name, self.nx, self.ny)),
                               device="cuda")

    def adjoint_view(self, name: str):
        """zero-copy torch view of an adjoint field (compact layout)"""
        import torch
        p = ctypes.c_void_p()
        n = ctypes.c_size_t(0)
        _check(lib().svof_adjoint_field(self._h, ADJ_FIELDS[name], ctypes.byref(p), ctypes.byref(n)))
        return torch.as_tensor(_DeviceArray(p.value, adjoint_shape(name, self.nx, self.ny)), device="cuda")

    def set_gravity(self, grav_vof: float, vof_ref: float):
        """the vof buoyancy extension on uy (absent from the reference; 0 = off)"""
        _check(lib().svof_set_gravity(self._h, float(grav_vof), float(vof_ref)))
        self.gravity = (float(grav_vof), float(vof_ref))

    def set_tension(self, tension: float):
        self.params.tension = float(tension)
        _check(lib().svof_set_params(self._h, ctypes.byref(self.params)))

    def tape_count(self) -> int:
        n = ctypes.c_size_t(0)
        _check(lib().svof_tape_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def integrate_fixed(self, dt: float, tape_ptr: int = 0):
        """one step with the given dt, enqueued; records the substep inputs at
        tape_ptr (device memory, tape_count() doubles) when non-zero"""
        _check(lib().svof_integrate_fixed(self._h, float(dt), ctypes.c_void_p(tape_ptr or None)))

    def adjoint_reset(self):
        _check(lib().svof_adjoint_reset(self._h))

    def adjoint_step(self, tape_ptr: int, dt: float):
        _check(lib().svof_adjoint_step(self._h, ctypes.c_void_p(tape_ptr), float(dt)))

    def adjoint_tension(self) -> float:
        out = ctypes.c_double(0.0)
        _check(lib().svof_adjoint_tension(self._h, ctypes.byref(out)))
        return out.value

    def adjoint_gravity(self) -> float:
        out = ctypes.c_double(0.0)
        _check(lib().svof_adjoint_gravity(self._h, ctypes.byref(out)))
        return out.value

    def adjoint_fluid_update_pressure(self, rk: int, dt: float):
        _check(lib().svof_adjoint_fluid_update_pressure(self._h, rk, dt))

    def adjoint_fluid_correct_velocity(self, rk: int, dt: float):
        _check(lib().svof_adjoint_fluid_correct_velocity(self._h, rk, dt))

    def adjoint_fluid_compute_potential(self, rk: int, dt: float):
        _check(lib().svof_adjoint_fluid_compute_potential(self._h, rk, dt))

    def adjoint_fluid_predict_field(self, rk: int, dt: float):
        _check(lib().svof_adjoint_fluid_predict_field(self._h, rk, dt))

    def adjoint_interface_update_vof(self, rk: int, dt: float):
        _check(lib().svof_adjoint_interface_update_vof(self._h, rk, dt))

    def adjoint_interface_compute_force(self):
        _check(lib().svof_adjoint_interface_compute_force(self._h))

    def adjoint_interface_compute_curvature_tensor(self):
        _check(lib().svof_adjoint_interface_compute_curvature_tensor(self._h))


# the 3D path (include/svof3d_b200.h)
from .solver3d import (EXPORTS3D, FIELDS3D, Solver3D, interior_shape3d, storage_shape3d)  # noqa: E402,F401
from .workloads import DROPLETS3D_ENV, InitialCondition3D, droplets3d  # noqa: E402,F401
