"""The 3D path of libsvof_b200.so through its C ABI (``include/svof3d_b200.h``).

:class:`Solver3D` mirrors the 2D :class:`simplevofsolver_b200.Solver`: the
reference's entry-point names (``fluid_decide_dt``,
``interface_compute_curvature_tensor``, ..., ``integrate``) with a third,
periodic z direction.  Storage shapes are (z, y, x[, comps]), x fastest.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import SvofError, lib
from .workloads import InitialCondition3D, read_npy_dir, write_npy_dir


class Params3D(ctypes.Structure):
    """svof3d_params_t"""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("m_dif", ctypes.c_double), ("t_dif", ctypes.c_double),
                ("tension", ctypes.c_double),
                ("coef_dt_adv", ctypes.c_double), ("coef_dt_dif", ctypes.c_double),
                ("add_buoyancy", ctypes.c_int),
                ("uy_xm", ctypes.c_double), ("uy_xp", ctypes.c_double),
                ("uz_xm", ctypes.c_double), ("uz_xp", ctypes.c_double),
                ("t_xm", ctypes.c_double), ("t_xp", ctypes.c_double),
                ("precision", ctypes.c_int)]


FP64, MIXED, MIXED_DC = 0, 1, 2
PRECISIONS = {"fp64": FP64, "mixed": MIXED, "mixed_dc": MIXED_DC}

FIELDS3D = {"ux": 0, "uy": 1, "uz": 2, "p": 3, "t": 4, "vof": 5, "psi": 6, "curv": 7, "normal": 8,
            "ifrcx": 9, "ifrcy": 10, "ifrcz": 11, "srcux_a": 12, "srcux_b": 13, "srcuy_a": 14, "srcuy_b": 15,
            "srcuz_a": 16, "srcuz_b": 17, "srct_a": 18, "srct_b": 19, "src_a": 20, "src_b": 21}

EXPORTS3D = ["svof3d_create", "svof3d_destroy", "svof3d_field_count", "svof3d_upload_field",
             "svof3d_download_field", "svof3d_device_field", "svof3d_load_interior", "svof3d_store_interior",
             "svof3d_load_interior_async", "svof3d_store_interior_async", "svof3d_io_wait",
             "svof3d_fluid_decide_dt", "svof3d_interface_compute_curvature_tensor",
             "svof3d_interface_compute_force", "svof3d_interface_update_vof", "svof3d_fluid_predict_field",
             "svof3d_fluid_compute_potential_dft", "svof3d_fluid_correct_velocity",
             "svof3d_fluid_update_pressure", "svof3d_integrate", "svof3d_run", "svof3d_enqueue_steps",
             "svof3d_last_dt", "svof3d_diagnostics", "svof3d_profile_step", "svof3d_synchronize", "svof3d_health",
             "svof3d_stream", "svof3d_last_error", "svof3d_statistics_collect", "svof3d_statistics_reset",
             "svof3d_statistics_count", "svof3d_statistics_reduce", "svof3d_statistics_field",
             "svof3d_set_tension", "svof3d_tape_count", "svof3d_integrate_fixed", "svof3d_adjoint_field",
             "svof3d_adjoint_reset", "svof3d_adjoint_step", "svof3d_adjoint_fluid_update_pressure",
             "svof3d_adjoint_fluid_correct_velocity", "svof3d_adjoint_fluid_compute_potential_dft",
             "svof3d_adjoint_fluid_predict_field", "svof3d_adjoint_interface_update_vof",
             "svof3d_adjoint_interface_compute_force", "svof3d_adjoint_interface_compute_curvature_tensor",
             "svof3d_adjoint_tension", "svof3d_set_gravity", "svof3d_adjoint_gravity",
             "svof3d_adjoint_set_gradient_floor", "svof3d_adjoint_set_precision"]

# adjoint fields (SVOF3_ADJ_*); compact layouts: ux faces (nz, ny, nx-1), cells (nz, ny, nx)
ADJ_FIELDS3D = {"ux": 0, "uy": 1, "uz": 2, "p": 3, "vof": 4, "psi": 5, "ifrcx": 6, "ifrcy": 7, "ifrcz": 8,
                "curv": 9, "normal": 10, "srcux_a": 11, "srcuy_a": 12, "srcuz_a": 13, "src_a": 14, "tension": 15,
                "gravity": 16}


def adjoint_shape3d(name: str, nx: int, ny: int, nz: int):
    if name in ("ux", "ifrcx", "srcux_a"):
        return (nz, ny, nx - 1)
    if name == "normal":
        return (nz, ny, nx, 4)
    return (nz, ny, nx)

# statistics quantities (SVOF3_STAT_*)
STAT_NAMES3D = ["ux1", "ux2", "uy1", "uy2", "uz1", "uz2", "t1", "t2", "uxt"]


def storage_shape3d(name: str, nx: int, ny: int, nz: int):
    if name == "ux":
        return (nz + 2, ny + 2, nx + 1)
    if name in ("uy", "uz", "p", "psi", "t", "curv"):
        return (nz + 2, ny + 2, nx + 2)
    if name == "vof":
        return (nz + 4, ny + 4, nx + 2)
    if name == "normal":
        return (nz + 2, ny + 2, nx, 4)
    if name in ("ifrcx", "srcux_a", "srcux_b"):
        return (nz, ny, nx - 1)
    if name in FIELDS3D:
        return (nz, ny, nx)
    raise KeyError(name)


def interior_shape3d(name: str, nx: int, ny: int, nz: int):
    return (nz, ny, nx + 1) if name == "ux" else (nz, ny, nx + 2)


_bound = False


def lib3() -> ctypes.CDLL:
    global _bound
    L = lib()
    if not _bound:
        vp, dp, sz, i, d = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
        pd = ctypes.POINTER(ctypes.c_double)
        L.svof3d_create.argtypes = [ctypes.POINTER(Params3D), dp, dp, ctypes.POINTER(vp)]
        L.svof3d_destroy.argtypes = [vp]
        L.svof3d_field_count.argtypes = [vp, i, ctypes.POINTER(sz)]
        for fn in ("svof3d_upload_field", "svof3d_download_field", "svof3d_load_interior", "svof3d_store_interior",
                   "svof3d_load_interior_async", "svof3d_store_interior_async"):
            getattr(L, fn).argtypes = [vp, i, dp, sz]
        L.svof3d_io_wait.argtypes = [vp]
        L.svof3d_statistics_collect.argtypes = [vp]
        L.svof3d_statistics_reset.argtypes = [vp]
        L.svof3d_statistics_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.svof3d_statistics_reduce.argtypes = [vp, i, dp, sz]
        L.svof3d_statistics_field.argtypes = [vp, i, dp, sz]
        L.svof3d_device_field.argtypes = [vp, i, ctypes.POINTER(vp)]
        L.svof3d_fluid_decide_dt.argtypes = [vp, pd]
        L.svof3d_interface_compute_curvature_tensor.argtypes = [vp]
        L.svof3d_interface_compute_force.argtypes = [vp]
        for fn in ("svof3d_interface_update_vof", "svof3d_fluid_predict_field", "svof3d_fluid_compute_potential_dft",
                   "svof3d_fluid_correct_velocity", "svof3d_fluid_update_pressure"):
            getattr(L, fn).argtypes = [vp, sz, d]
        L.svof3d_integrate.argtypes = [vp, pd]
        L.svof3d_run.argtypes = [vp, i, dp]
        L.svof3d_enqueue_steps.argtypes = [vp, i]
        L.svof3d_last_dt.argtypes = [vp, pd]
        L.svof3d_diagnostics.argtypes = [vp, pd, pd, pd, pd]
        L.svof3d_profile_step.argtypes = [vp, dp, dp, i]
        L.svof3d_synchronize.argtypes = [vp]
        L.svof3d_health.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong),
                                    ctypes.c_int]
        L.svof3d_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.svof3d_last_error.restype = ctypes.c_char_p
        L.svof3d_set_tension.argtypes = [vp, d]
        L.svof3d_tape_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.svof3d_integrate_fixed.argtypes = [vp, d, vp]
        L.svof3d_adjoint_field.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        L.svof3d_adjoint_reset.argtypes = [vp]
        L.svof3d_adjoint_step.argtypes = [vp, vp, d]
        for fn in ("svof3d_adjoint_fluid_update_pressure", "svof3d_adjoint_fluid_correct_velocity",
                   "svof3d_adjoint_fluid_compute_potential_dft", "svof3d_adjoint_fluid_predict_field",
                   "svof3d_adjoint_interface_update_vof"):
            getattr(L, fn).argtypes = [vp, sz, d]
        L.svof3d_adjoint_interface_compute_force.argtypes = [vp]
        L.svof3d_adjoint_interface_compute_curvature_tensor.argtypes = [vp]
        L.svof3d_adjoint_tension.argtypes = [vp, pd]
        L.svof3d_set_gravity.argtypes = [vp, d, d]
        L.svof3d_adjoint_gravity.argtypes = [vp, pd]
        L.svof3d_adjoint_set_gradient_floor.argtypes = [vp, d]
        L.svof3d_adjoint_set_precision.argtypes = [vp, i]
        _bound = True
    return L


def _check(rc: int):
    if rc != 0:
        raise SvofError(lib3().svof3d_last_error().decode())


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Solver3D:
    """One 3D domain on the GPU (FP64).  ``physical`` as for the 2D Solver."""

    KERNEL_KINDS = ["dt", "geom", "force", "vof", "predict", "poisson_fwd", "poisson_z", "poisson_solve",
                    "poisson_inv", "project"]

    def __init__(self, ic: InitialCondition3D, physical: dict, add_buoyancy: bool = False,
                 uy_walls=(0.0, 0.0), uz_walls=(0.0, 0.0), t_walls=(0.0, 0.0), precision: str = "fp64"):
        """precision: "fp64", "mixed" or "mixed_dc" (see svof3d_b200.h)"""
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be 'fp64', 'mixed' or 'mixed_dc', not {precision!r}")
        L = lib3()
        self.precision = precision
        self.nx, self.ny, self.nz = int(ic.nx), int(ic.ny), int(ic.nz)
        self.params = Params3D(self.nx, self.ny, self.nz, float(ic.lx), float(ic.ly), float(ic.lz),
                               physical["m_dif"], physical["t_dif"], physical["tension"],
                               physical["coef_dt_adv"], physical["coef_dt_dif"], int(bool(add_buoyancy)),
                               float(uy_walls[0]), float(uy_walls[1]), float(uz_walls[0]), float(uz_walls[1]),
                               float(t_walls[0]), float(t_walls[1]), PRECISIONS[precision])
        self.gravity = (0.0, 0.0)
        self._h = ctypes.c_void_p()
        self._io_held = []
        xf, xc = _c(ic.xf), _c(ic.xc)
        self._grid = (float(ic.lx), float(ic.ly), float(ic.lz), xf.copy(), xc.copy())
        _check(L.svof3d_create(ctypes.byref(self.params), xf.ctypes.data, xc.ctypes.data, ctypes.byref(self._h)))
        for k, v in ic.fields().items():
            self.load_interior(k, v)

    @classmethod
    def from_npy_dir(cls, dirname: str, physical: dict, **kw):
        """restart from a 3D directory in the save layout; returns (solver,
        step, time)"""
        ic = read_npy_dir(dirname)
        if not isinstance(ic, InitialCondition3D):
            raise ValueError(f"{dirname} holds a 2D restart set")
        step = int(np.load(os.path.join(dirname, "step.npy")))
        time = float(np.load(os.path.join(dirname, "time.npy")))
        return cls(ic, physical, **kw), step, time

    # ------------------------------------------------------------ restart files
    def state(self) -> InitialCondition3D:
        """the current fields in the restart layout, with the grid"""
        lx, ly, lz, xf, xc = self._grid
        return InitialCondition3D(self.nx, self.ny, self.nz, lx, ly, lz, xf.copy(), xc.copy(),
                                  *(self.interior(k) for k in ("ux", "uy", "uz", "p", "t", "vof")))

    def fluid_save(self, dirname: str):
        """m_dif, t_dif and ux, uy, uz, p, t (src/fluid/save.c with uz)"""
        os.makedirs(dirname, exist_ok=True)
        np.save(os.path.join(dirname, "m_dif.npy"), np.array(self.params.m_dif))
        np.save(os.path.join(dirname, "t_dif.npy"), np.array(self.params.t_dif))
        for k in ("ux", "uy", "uz", "p", "t"):
            np.save(os.path.join(dirname, f"{k}.npy"), self.interior(k))

    def interface_save(self, dirname: str):
        """surface_tension and vof (src/interface/save.c)"""
        os.makedirs(dirname, exist_ok=True)
        np.save(os.path.join(dirname, "surface_tension.npy"), np.array(self.params.tension))
        np.save(os.path.join(dirname, "vof.npy"), self.interior("vof"))

    def save(self, dirname: str, step: int = 0, time: float = 0.0):
        """a save / restart directory: step, time, the grid, fluid and interface"""
        write_npy_dir(self.state(), dirname, step, time)
        self.fluid_save(dirname)
        self.interface_save(dirname)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib3().svof3d_destroy(self._h)  # waits for queued copies first
            self._h = ctypes.c_void_p()
            self._io_held = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _shape(self, name):
        return storage_shape3d(name, self.nx, self.ny, self.nz)

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self._shape(name))
        _check(lib3().svof3d_download_field(self._h, FIELDS3D[name], out.ctypes.data, out.size))
        return out

    def set_field(self, name: str, a: np.ndarray):
        a = _c(a)
        if a.shape != self._shape(name):
            raise ValueError(f"{name}: expected shape {self._shape(name)}, got {a.shape}")
        _check(lib3().svof3d_upload_field(self._h, FIELDS3D[name], a.ctypes.data, a.size))

    def load_interior(self, name: str, a: np.ndarray):
        a = _c(a)
        want = interior_shape3d(name, self.nx, self.ny, self.nz)
        if a.shape != want:
            raise ValueError(f"{name}: expected shape {want}, got {a.shape}")
        _check(lib3().svof3d_load_interior(self._h, FIELDS3D[name], a.ctypes.data, a.size))

    def interior(self, name: str) -> np.ndarray:
        out = np.empty(interior_shape3d(name, self.nx, self.ny, self.nz))
        _check(lib3().svof3d_store_interior(self._h, FIELDS3D[name], out.ctypes.data, out.size))
        return out

    def load_interior_async(self, name: str, a: np.ndarray):
        """Queue a restart-layout load; `a` (page-locked for overlap) is held
        until io_wait()."""
        a = _c(a)
        want = interior_shape3d(name, self.nx, self.ny, self.nz)
        if a.shape != want:
            raise ValueError(f"{name}: expected shape {want}, got {a.shape}")
        _check(lib3().svof3d_load_interior_async(self._h, FIELDS3D[name], a.ctypes.data, a.size))
        self._io_held.append(a)

    def store_interior_async(self, name: str, out: np.ndarray):
        """Queue a restart-layout store into `out`, a C-contiguous float64
        array of the field's restart shape, complete after io_wait()."""
        want = interior_shape3d(name, self.nx, self.ny, self.nz)
        if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != want
                or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError(f"{name}: expected a writeable C-contiguous float64 array of shape {want}")
        _check(lib3().svof3d_store_interior_async(self._h, FIELDS3D[name], out.ctypes.data, out.size))
        self._io_held.append(out)

    def io_wait(self):
        """Wait for every queued load, step and store."""
        _check(lib3().svof3d_io_wait(self._h))
        self._io_held.clear()

    def device_ptr(self, name: str) -> int:
        p = ctypes.c_void_p()
        _check(lib3().svof3d_device_field(self._h, FIELDS3D[name], ctypes.byref(p)))
        return int(p.value)

    def stream(self) -> int:
        p = ctypes.c_void_p()
        _check(lib3().svof3d_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    # ------------------------------------------------------------ step functions
    def fluid_decide_dt(self) -> float:
        dt = ctypes.c_double(0.0)
        _check(lib3().svof3d_fluid_decide_dt(self._h, ctypes.byref(dt)))
        return dt.value

    def interface_compute_curvature_tensor(self):
        _check(lib3().svof3d_interface_compute_curvature_tensor(self._h))

    def interface_compute_force(self):
        _check(lib3().svof3d_interface_compute_force(self._h))

    def interface_update_vof(self, rkstep: int, dt: float):
        _check(lib3().svof3d_interface_update_vof(self._h, rkstep, dt))

    def fluid_predict_field(self, rkstep: int, dt: float):
        _check(lib3().svof3d_fluid_predict_field(self._h, rkstep, dt))

    def fluid_compute_potential_dft(self, rkstep: int, dt: float):
        _check(lib3().svof3d_fluid_compute_potential_dft(self._h, rkstep, dt))

    fluid_compute_potential = fluid_compute_potential_dft

    def fluid_correct_velocity(self, rkstep: int, dt: float):
        _check(lib3().svof3d_fluid_correct_velocity(self._h, rkstep, dt))

    def fluid_update_pressure(self, rkstep: int, dt: float):
        _check(lib3().svof3d_fluid_update_pressure(self._h, rkstep, dt))

    def integrate(self) -> float:
        dt = ctypes.c_double(0.0)
        _check(lib3().svof3d_integrate(self._h, ctypes.byref(dt)))
        return dt.value

    def run(self, nsteps: int) -> np.ndarray:
        dts = np.zeros(max(int(nsteps), 1))
        _check(lib3().svof3d_run(self._h, int(nsteps), dts.ctypes.data))
        return dts[:nsteps]

    def enqueue_steps(self, nsteps: int):
        _check(lib3().svof3d_enqueue_steps(self._h, int(nsteps)))

    def last_dt(self) -> float:
        dt = ctypes.c_double(0.0)
        _check(lib3().svof3d_last_dt(self._h, ctypes.byref(dt)))
        return dt.value

    def diagnostics(self) -> dict:
        v = [ctypes.c_double() for _ in range(4)]
        _check(lib3().svof3d_diagnostics(self._h, *[ctypes.byref(x) for x in v]))
        return dict(divmax=v[0].value, vofmin=v[1].value, vofmax=v[2].value, volume=v[3].value)

    def profile_step(self) -> dict:
        n = len(self.KERNEL_KINDS)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int32)
        _check(lib3().svof3d_profile_step(self._h, ms.ctypes.data, cnt.ctypes.data, n))
        return {k: (float(ms[q]), int(cnt[q])) for q, k in enumerate(self.KERNEL_KINDS)}

    # ------------------------------------------------- time-averaged statistics
    def statistics_collect(self):
        """add one sample of the current fields to the device accumulators;
        queued, does not wait"""
        _check(lib3().svof3d_statistics_collect(self._h))

    def statistics_reset(self):
        _check(lib3().svof3d_statistics_reset(self._h))

    def statistics_count(self) -> int:
        n = ctypes.c_size_t(0)
        _check(lib3().svof3d_statistics_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def statistics_reduced(self) -> dict:
        """the y-z sums of every quantity (one vector along x each), plus 'num'"""
        out = {}
        for q, k in enumerate(STAT_NAMES3D):
            v = np.zeros(self.nx + (1 if k in ("ux1", "ux2", "uxt") else 2))
            _check(lib3().svof3d_statistics_reduce(self._h, q, v.ctypes.data, v.size))
            out[k] = v
        out["num"] = self.statistics_count()
        return out

    def statistics_field(self, name: str) -> np.ndarray:
        """the accumulated array of one quantity, nz x ny x (nx+1) or nz x ny x (nx+2)"""
        q = STAT_NAMES3D.index(name)
        v = np.zeros((self.nz, self.ny, self.nx + (1 if name in ("ux1", "ux2", "uxt") else 2)))
        _check(lib3().svof3d_statistics_field(self._h, q, v.ctypes.data, v.size))
        return v

    def synchronize(self):
        _check(lib3().svof3d_synchronize(self._h))

    def health(self, reset=False):
        """the device health counters since creation or the last reset:
        {"newton_unconverged": THINC intercepts whose Newton iteration missed
        its tolerance, "small_pivots": Poisson x line solves (other than the
        singular ky = kz = 0 line) that met a pivot <= DBL_EPSILON}"""
        a, b = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
        _check(lib3().svof3d_health(self._h, ctypes.byref(a), ctypes.byref(b), 1 if reset else 0))
        return {"newton_unconverged": a.value, "small_pivots": b.value}

    # ------------------------------------------------------------ differentiation form
    def device_view(self, name: str):
        """zero-copy torch view of a field's current device storage (valid
        until the next call that swaps its buffers; synchronise the solver's
        stream and torch's around its use)"""
        import torch
        from . import _DeviceArray
        return torch.as_tensor(_DeviceArray(self.device_ptr(name), storage_shape3d(name, self.nx, self.ny, self.nz)),
                               device="cuda")

    def adjoint_view(self, name: str):
        """zero-copy torch view of an adjoint field (compact layout)"""
        import torch
        from . import _DeviceArray
        p = ctypes.c_void_p()
        n = ctypes.c_size_t(0)
        _check(lib3().svof3d_adjoint_field(self._h, ADJ_FIELDS3D[name], ctypes.byref(p), ctypes.byref(n)))
        return torch.as_tensor(_DeviceArray(p.value, adjoint_shape3d(name, self.nx, self.ny, self.nz)),
                               device="cuda")

    def set_tension(self, tension: float):
        _check(lib3().svof3d_set_tension(self._h, float(tension)))
        self.params.tension = float(tension)

    def set_gravity(self, grav_vof: float, vof_ref: float):
        """the vof buoyancy extension on uy (absent from the reference; 0 = off)"""
        _check(lib3().svof3d_set_gravity(self._h, float(grav_vof), float(vof_ref)))
        self.gravity = (float(grav_vof), float(vof_ref))

    def tape_count(self) -> int:
        n = ctypes.c_size_t(0)
        _check(lib3().svof3d_tape_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def integrate_fixed(self, dt: float, tape_ptr: int = 0):
        """one step with the given dt, enqueued; records the substep inputs at
        tape_ptr (device memory, tape_count() doubles) when non-zero"""
        _check(lib3().svof3d_integrate_fixed(self._h, float(dt), ctypes.c_void_p(tape_ptr or None)))

    def adjoint_reset(self):
        _check(lib3().svof3d_adjoint_reset(self._h))

    def adjoint_set_precision(self, precision: str):
        """"fp64" (default) or "fp32": the storage of the adjoint's
        intermediates (the state's adjoints, accumulators, arithmetic, line
        recurrences and Poisson solve stay FP64); discards the adjoint's
        buffers when it changes"""
        if precision not in ("fp64", "fp32"):
            raise ValueError(f"adjoint precision must be 'fp64' or 'fp32', not {precision!r}")
        _check(lib3().svof3d_adjoint_set_precision(self._h, int(precision == "fp32")))

    def adjoint_set_gradient_floor(self, tau: float):
        """corners flatter than tau (vof variation across a cell) have no
        normal derivative in the adjoint; 0 = exact (the FP64 default), 1e-5
        the mixed paths' default"""
        _check(lib3().svof3d_adjoint_set_gradient_floor(self._h, float(tau)))

    def adjoint_step(self, tape_ptr: int, dt: float):
        _check(lib3().svof3d_adjoint_step(self._h, ctypes.c_void_p(tape_ptr), float(dt)))

    def adjoint_tension(self) -> float:
        out = ctypes.c_double(0.0)
        _check(lib3().svof3d_adjoint_tension(self._h, ctypes.byref(out)))
        return out.value

    def adjoint_gravity(self) -> float:
        out = ctypes.c_double(0.0)
        _check(lib3().svof3d_adjoint_gravity(self._h, ctypes.byref(out)))
        return out.value

    def adjoint_fluid_update_pressure(self, rk: int, dt: float):
        _check(lib3().svof3d_adjoint_fluid_update_pressure(self._h, rk, dt))

    def adjoint_fluid_correct_velocity(self, rk: int, dt: float):
        _check(lib3().svof3d_adjoint_fluid_correct_velocity(self._h, rk, dt))

    def adjoint_fluid_compute_potential_dft(self, rk: int, dt: float):
        _check(lib3().svof3d_adjoint_fluid_compute_potential_dft(self._h, rk, dt))

    def adjoint_fluid_predict_field(self, rk: int, dt: float):
        _check(lib3().svof3d_adjoint_fluid_predict_field(self._h, rk, dt))

    def adjoint_interface_update_vof(self, rk: int, dt: float):
        _check(lib3().svof3d_adjoint_interface_update_vof(self._h, rk, dt))

    def adjoint_interface_compute_force(self):
        _check(lib3().svof3d_adjoint_interface_compute_force(self._h))

    def adjoint_interface_compute_curvature_tensor(self):
        _check(lib3().svof3d_adjoint_interface_compute_curvature_tensor(self._h))
