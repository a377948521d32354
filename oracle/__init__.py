"""Oracle for the CUDA path: ctypes front-ends of two CPU libraries.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg (and its ``--impl reference`` arm) import this
package; the product library never does.

* :class:`Oracle` drives ``libsvof_oracle.so``, this repository's C
  restatement of the reference algorithm (``oracle/svof_oracle.c``);
  :class:`Oracle3D` its 3D extension (``oracle/svof_oracle3d.c``).
* :func:`run_reference` drives ``_ref/libsvof_ref[_c0].so``, the reference's
  own ``src/*.c`` compiled against single-rank shims, in a fresh process (the
  reference keeps solver state in process-wide statics).

Storage layouts are the reference's (``include/array_macros/``): x fastest,
x ghost cells and y halo rows included.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libsvof_oracle.so")
REF_LIBS = {"ref": os.path.join(HERE, "_ref", "libsvof_ref.so"),
            "c0": os.path.join(HERE, "_ref", "libsvof_ref_c0.so")}

# halo rows per field (y) and storage shape (rows, cols[, comps]) for nx, ny
NHALO = {"ux": 1, "uy": 1, "p": 1, "psi": 1, "t": 1, "vof": 2, "curv": 1}


def storage_shape(name: str, nx: int, ny: int):
    if name == "ux":
        return (ny + 2, nx + 1)
    if name in ("uy", "p", "psi", "t", "curv"):
        return (ny + 2, nx + 2)
    if name == "vof":
        return (ny + 4, nx + 2)
    if name == "dvof":
        return (ny + 3, nx + 1, 2)
    if name == "normal":
        return (ny + 2, nx, 3)
    if name == "flxx":
        return (ny, nx + 1)
    if name == "flxy":
        return (ny + 1, nx)
    if name in ("ifrcx",) or name.startswith("srcux"):
        return (ny, nx - 1)
    if name in ("ifrcy", "src0", "src1") or name.startswith("srcuy") or name.startswith("srct"):
        return (ny, nx)
    raise KeyError(name)


def interior_rows(name: str, arr: np.ndarray, ny: int) -> np.ndarray:
    """rows j = 1..ny of a halo'd field (the part the NPY restart files hold)"""
    h = NHALO[name]
    return arr[h:h + ny]


class _Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("m_dif", ctypes.c_double), ("t_dif", ctypes.c_double),
                ("tension", ctypes.c_double),
                ("coef_dt_adv", ctypes.c_double), ("coef_dt_dif", ctypes.c_double),
                ("add_buoyancy", ctypes.c_int),
                ("uy_xm", ctypes.c_double), ("uy_xp", ctypes.c_double),
                ("t_xm", ctypes.c_double), ("t_xp", ctypes.c_double)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} missing: run 'make -C oracle oracle'")
        L = ctypes.CDLL(ORACLE_LIB)
        L.svo_create.restype = ctypes.c_void_p
        L.svo_create.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_void_p]
        L.svo_destroy.argtypes = [ctypes.c_void_p]
        L.svo_field.restype = ctypes.POINTER(ctypes.c_double)
        L.svo_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        for fn in ("svo_init_boundaries", "svo_curvature_tensor", "svo_force", "svo_x_grid_is_uniform"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.svo_decide_dt.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        for fn in ("svo_update_vof", "svo_predict", "svo_potential_dct", "svo_potential_dft",
                   "svo_correct", "svo_update_pressure"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.svo_integrate.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.svo_integrate_fixed.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.svo_set_gravity.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.svo_tl_integrate_fixed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double]
        L.svo_tl_curvature_tensor.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.svo_tl_force.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
        L.svo_tl_update_vof.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.svo_tl_predict.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.svo_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.svo_logging.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.svo_stat_collect.argtypes = [ctypes.c_void_p]
        L.svo_stat_reduce.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.svo_stat_num.argtypes = [ctypes.c_void_p]
        L.svo_stat_num.restype = ctypes.c_long
        _lib = L
    return _lib


FIELD_NAMES = ["ux", "uy", "p", "psi", "t", "srcux0", "srcux1", "srcux2", "srcuy0", "srcuy1",
               "srcuy2", "srct0", "srct1", "srct2", "vof", "ifrcx", "ifrcy", "dvof", "normal",
               "curv", "flxx", "flxy", "src0", "src1"]


class Oracle:
    """The C restatement, 2D FP64.  ``params`` holds m_dif, t_dif, tension,
    coef_dt_adv, coef_dt_dif (see simplevofsolver_b200.workloads.physical_params)."""

    def __init__(self, ic, params: dict, add_buoyancy: bool = False,
                 uy_walls=(0.0, 0.0), t_walls=(0.0, 0.0)):
        L = _load()
        self.nx, self.ny = int(ic.nx), int(ic.ny)
        pr = _Params(self.nx, self.ny, float(ic.lx), float(ic.ly), params["m_dif"], params["t_dif"],
                     params["tension"], params["coef_dt_adv"], params["coef_dt_dif"],
                     int(bool(add_buoyancy)), float(uy_walls[0]), float(uy_walls[1]),
                     float(t_walls[0]), float(t_walls[1]))
        xf = np.ascontiguousarray(ic.xf, dtype=np.float64)
        xc = np.ascontiguousarray(ic.xc, dtype=np.float64)
        # kept for tangent contexts on the same grid (wall values zero)
        self._grid = (pr, xf, xc)
        self._h = L.svo_create(ctypes.byref(pr), xf.ctypes.data, xc.ctypes.data)
        if not self._h:
            raise ValueError("svo_create failed")
        for k, v in ic.fields().items():
            interior_rows(k, self.field(k), self.ny)[...] = v
        L.svo_init_boundaries(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            _load().svo_destroy(self._h)
            self._h = None

    def field(self, name: str) -> np.ndarray:
        """live view of a field's storage"""
        n = ctypes.c_long(0)
        ptr = _load().svo_field(self._h, name.encode(), ctypes.byref(n))
        if not ptr:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).reshape(storage_shape(name, self.nx, self.ny))

    def snapshot(self, names=("ux", "uy", "p", "psi", "t", "vof")):
        return {k: self.field(k).copy() for k in names}

    @property
    def uniform(self):
        return bool(_load().svo_x_grid_is_uniform(self._h))

    def decide_dt(self):
        dt = ctypes.c_double(0.0)
        _load().svo_decide_dt(self._h, ctypes.byref(dt))
        return dt.value

    def curvature_tensor(self):
        _load().svo_curvature_tensor(self._h)

    def force(self):
        _load().svo_force(self._h)

    def update_vof(self, rk, dt):
        _load().svo_update_vof(self._h, rk, dt)

    def predict(self, rk, dt):
        _load().svo_predict(self._h, rk, dt)

    def potential(self, rk, dt):
        if self.uniform:
            _load().svo_potential_dct(self._h, rk, dt)
        else:
            _load().svo_potential_dft(self._h, rk, dt)

    def correct(self, rk, dt):
        _load().svo_correct(self._h, rk, dt)

    def update_pressure(self, rk, dt):
        _load().svo_update_pressure(self._h, rk, dt)

    def integrate_fixed(self, dt: float):
        """one step with the given dt (no CFL decision)"""
        _load().svo_integrate_fixed(self._h, float(dt))

    def set_gravity(self, grav_vof: float, vof_ref: float):
        """the vof buoyancy extension (absent from the reference): srcuy +=
        grav_vof * (vof at the uy face - vof_ref)"""
        _load().svo_set_gravity(self._h, float(grav_vof), float(vof_ref))

    def tangent(self) -> "OracleTangent":
        """a zero tangent of this context (tangent-linear model)"""
        return OracleTangent(self)

    def run(self, nsteps: int) -> np.ndarray:
        dts = np.zeros(max(nsteps, 1))
        if _load().svo_run(self._h, int(nsteps), dts.ctypes.data) != 0:
            raise RuntimeError("svo_run failed")
        return dts[:nsteps]

    LOGGING_NAMES = ["momentum_x", "momentum_y", "energy_ux", "energy_uy", "energy_t", "nu_heat_flux",
                     "nu_kinetic_injection", "nu_kinetic_dissipation", "nu_thermal_dissipation"]

    def logging(self) -> dict:
        """src/logging/momentum.c, energy.c and nusselt/ on the current fields
        (svo_logging: the reference's loops and order)"""
        out = np.zeros(9)
        _load().svo_logging(self._h, out.ctypes.data)
        return dict(zip(self.LOGGING_NAMES, out.tolist()))

    STAT_NAMES = ["ux1", "ux2", "uy1", "uy2", "t1", "t2", "uxt"]

    def statistics_collect(self):
        """one sample of src/statistics.c:117-204 (svo_stat_collect)"""
        _load().svo_stat_collect(self._h)

    def statistics_reduced(self) -> dict:
        """reduce_and_write's row sums (src/statistics.c:232-281) of every
        quantity, plus 'num' the number of samples"""
        out = {}
        for q, k in enumerate(self.STAT_NAMES):
            v = np.zeros(self.nx + (1 if k in ("ux1", "ux2", "uxt") else 2))
            _load().svo_stat_reduce(self._h, q, v.ctypes.data)
            out[k] = v
        out["num"] = int(_load().svo_stat_num(self._h))
        return out


# ---------------------------------------------------------------- 3D

class OracleTangent:
    """Tangents of an :class:`Oracle`'s fields (svof_oracle_tl.inc): a second
    context on the same grid with zero wall values.  ``step`` advances the
    primal and the tangent by one step of the tangent-linear model with the
    time step held fixed."""

    def __init__(self, primal: Oracle):
        L = _load()
        pr, xf, xc = primal._grid
        z = _Params(pr.nx, pr.ny, pr.lx, pr.ly, pr.m_dif, pr.t_dif, pr.tension, pr.coef_dt_adv,
                    pr.coef_dt_dif, pr.add_buoyancy, 0.0, 0.0, 0.0, 0.0)
        self.primal = primal
        self.nx, self.ny = primal.nx, primal.ny
        self._h = L.svo_create(ctypes.byref(z), xf.ctypes.data, xc.ctypes.data)
        if not self._h:
            raise ValueError("svo_create failed")

    def __del__(self):
        if getattr(self, "_h", None):
            _load().svo_destroy(self._h)
            self._h = None

    def field(self, name: str) -> np.ndarray:
        n = ctypes.c_long(0)
        ptr = _load().svo_field(self._h, name.encode(), ctypes.byref(n))
        if not ptr:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).reshape(storage_shape(name, self.nx, self.ny))

    def init_boundaries(self):
        _load().svo_init_boundaries(self._h)

    def step(self, dt: float, dtension: float = 0.0, dgrav: float = 0.0):
        _load().svo_tl_integrate_fixed(self.primal._h, self._h, float(dt), float(dtension), float(dgrav))

    # the linearised functions one by one (each before the primal function)
    def curvature_tensor(self):
        _load().svo_tl_curvature_tensor(self.primal._h, self._h)

    def force(self, dtension: float = 0.0):
        _load().svo_tl_force(self.primal._h, self._h, float(dtension))

    def update_vof(self, rk, dt):
        _load().svo_tl_update_vof(self.primal._h, self._h, int(rk), float(dt))

    def predict(self, rk, dt, dgrav: float = 0.0):
        _load().svo_tl_predict(self.primal._h, self._h, int(rk), float(dt), float(dgrav))

    def potential(self, rk, dt):
        f = _load().svo_potential_dct if self.primal.uniform else _load().svo_potential_dft
        f(self._h, int(rk), float(dt))

    def correct(self, rk, dt):
        _load().svo_correct(self._h, int(rk), float(dt))

    def update_pressure(self, rk, dt):
        _load().svo_update_pressure(self._h, int(rk), float(dt))


def storage_shape3d(name: str, nx: int, ny: int, nz: int):
    """storage shapes of the 3D restatement (z, y, x[, comps]), x fastest"""
    if name == "ux":
        return (nz + 2, ny + 2, nx + 1)
    if name in ("uy", "uz", "p", "psi", "t", "curv"):
        return (nz + 2, ny + 2, nx + 2)
    if name == "vof":
        return (nz + 4, ny + 4, nx + 2)
    if name == "dvof":
        return (nz + 3, ny + 3, nx + 1, 3)
    if name == "normal":
        return (nz + 2, ny + 2, nx, 4)
    if name == "ifrcx" or name.startswith("srcux"):
        return (nz, ny, nx - 1)
    if name in ("ifrcy", "ifrcz", "src0", "src1") or name[:5] in ("srcuy", "srcuz") or name.startswith("srct"):
        return (nz, ny, nx)
    raise KeyError(name)


NHALO3D = {"ux": 1, "uy": 1, "uz": 1, "p": 1, "psi": 1, "t": 1, "vof": 2, "curv": 1}


def interior3d(name: str, arr: np.ndarray, ny: int, nz: int) -> np.ndarray:
    """the j = 1..ny, k = 1..nz part of a halo'd 3D field"""
    h = NHALO3D[name]
    return arr[h:h + nz, h:h + ny]


class _Params3D(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("m_dif", ctypes.c_double), ("t_dif", ctypes.c_double),
                ("tension", ctypes.c_double),
                ("coef_dt_adv", ctypes.c_double), ("coef_dt_dif", ctypes.c_double),
                ("add_buoyancy", ctypes.c_int),
                ("uy_xm", ctypes.c_double), ("uy_xp", ctypes.c_double),
                ("uz_xm", ctypes.c_double), ("uz_xp", ctypes.c_double),
                ("t_xm", ctypes.c_double), ("t_xp", ctypes.c_double)]


_lib3 = None


def _load3():
    global _lib3
    if _lib3 is None:
        L = _load()
        L.svo3_create.restype = ctypes.c_void_p
        L.svo3_create.argtypes = [ctypes.POINTER(_Params3D), ctypes.c_void_p, ctypes.c_void_p]
        L.svo3_destroy.argtypes = [ctypes.c_void_p]
        L.svo3_field.restype = ctypes.POINTER(ctypes.c_double)
        L.svo3_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        for fn in ("svo3_init_boundaries", "svo3_curvature_tensor", "svo3_force"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.svo3_decide_dt.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        for fn in ("svo3_update_vof", "svo3_predict", "svo3_potential", "svo3_correct", "svo3_update_pressure"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.svo3_integrate.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.svo3_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.svo3_set_gravity.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.svo3_stat_collect.argtypes = [ctypes.c_void_p]
        L.svo3_stat_reduce.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.svo3_stat_num.argtypes = [ctypes.c_void_p]
        L.svo3_stat_num.restype = ctypes.c_long
        _lib3 = L
    return _lib3


FIELD_NAMES3D = ["ux", "uy", "uz", "p", "psi", "t", "vof", "curv", "normal", "dvof", "ifrcx", "ifrcy", "ifrcz",
                 "srcux0", "srcuy0", "srcuz0", "srct0", "srcux1", "srcuy1", "srcuz1", "srct1", "src0", "src1"]


class Oracle3D:
    """The 3D C restatement (oracle/svof_oracle3d.c), FP64.  ``ic`` is a
    simplevofsolver_b200.workloads.InitialCondition3D."""

    def __init__(self, ic, params: dict, add_buoyancy: bool = False, uy_walls=(0.0, 0.0),
                 uz_walls=(0.0, 0.0), t_walls=(0.0, 0.0)):
        L = _load3()
        self.nx, self.ny, self.nz = int(ic.nx), int(ic.ny), int(ic.nz)
        pr = _Params3D(self.nx, self.ny, self.nz, float(ic.lx), float(ic.ly), float(ic.lz),
                       params["m_dif"], params["t_dif"], params["tension"], params["coef_dt_adv"],
                       params["coef_dt_dif"], int(bool(add_buoyancy)), float(uy_walls[0]),
                       float(uy_walls[1]), float(uz_walls[0]), float(uz_walls[1]), float(t_walls[0]),
                       float(t_walls[1]))
        xf = np.ascontiguousarray(ic.xf, dtype=np.float64)
        xc = np.ascontiguousarray(ic.xc, dtype=np.float64)
        self._h = L.svo3_create(ctypes.byref(pr), xf.ctypes.data, xc.ctypes.data)
        if not self._h:
            raise ValueError("svo3_create failed")
        for k, v in ic.fields().items():
            interior3d(k, self.field(k), self.ny, self.nz)[...] = v
        L.svo3_init_boundaries(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            _load3().svo3_destroy(self._h)
            self._h = None

    def field(self, name: str) -> np.ndarray:
        n = ctypes.c_long(0)
        ptr = _load3().svo3_field(self._h, name.encode(), ctypes.byref(n))
        if not ptr:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).reshape(
            storage_shape3d(name, self.nx, self.ny, self.nz))

    def snapshot(self, names=("ux", "uy", "uz", "p", "psi", "t", "vof")):
        return {k: self.field(k).copy() for k in names}

    def decide_dt(self):
        dt = ctypes.c_double(0.0)
        _load3().svo3_decide_dt(self._h, ctypes.byref(dt))
        return dt.value

    def curvature_tensor(self):
        _load3().svo3_curvature_tensor(self._h)

    def force(self):
        _load3().svo3_force(self._h)

    def update_vof(self, rk, dt):
        _load3().svo3_update_vof(self._h, rk, dt)

    def predict(self, rk, dt):
        _load3().svo3_predict(self._h, rk, dt)

    def potential(self, rk, dt):
        _load3().svo3_potential(self._h, rk, dt)

    def correct(self, rk, dt):
        _load3().svo3_correct(self._h, rk, dt)

    def update_pressure(self, rk, dt):
        _load3().svo3_update_pressure(self._h, rk, dt)

    def set_gravity(self, grav_vof: float, vof_ref: float):
        """the vof buoyancy extension on uy (0 = off)"""
        _load3().svo3_set_gravity(self._h, float(grav_vof), float(vof_ref))

    def substeps(self, dt):
        """one step's three Runge-Kutta substeps with a given dt"""
        for rk in range(3):
            self.curvature_tensor()
            self.force()
            self.update_vof(rk, dt)
            self.predict(rk, dt)
            self.potential(rk, dt)
            self.correct(rk, dt)
            self.update_pressure(rk, dt)

    def run(self, nsteps: int) -> np.ndarray:
        dts = np.zeros(max(nsteps, 1))
        if _load3().svo3_run(self._h, int(nsteps), dts.ctypes.data) != 0:
            raise RuntimeError("svo3_run failed")
        return dts[:nsteps]

    STAT_NAMES = ["ux1", "ux2", "uy1", "uy2", "uz1", "uz2", "t1", "t2", "uxt"]

    def statistics_collect(self):
        """one sample of the statistics (svo3_stat_collect)"""
        _load3().svo3_stat_collect(self._h)

    def statistics_reduced(self) -> dict:
        """the y-z sums of every quantity, plus 'num'"""
        out = {}
        for q, k in enumerate(self.STAT_NAMES):
            v = np.zeros(self.nx + (1 if k in ("ux1", "ux2", "uxt") else 2))
            _load3().svo3_stat_reduce(self._h, q, v.ctypes.data)
            out[k] = v
        out["num"] = int(_load3().svo3_stat_num(self._h))
        return out


# ---------------------------------------------------------------- reference

def reference_available(variant: str = "c0") -> bool:
    return os.path.exists(REF_LIBS[variant])


def run_reference(ic, env: dict, nsteps: int, variant: str = "c0",
                  names=("ux", "uy", "p", "psi", "t", "vof"), timeout: float = 1800.0):
    """Run the compiled reference for ``nsteps`` steps from ``ic`` (written to a
    temporary NPY directory and read back by the reference's own fluid_init /
    interface_init) in a fresh Python process (``oracle/_ref_runner.py``).
    Returns {name: storage array (reshaped), 'dts': ..., 'seconds': ...}."""
    import subprocess
    import sys
    from simplevofsolver_b200.workloads import write_npy_dir
    if not reference_available(variant):
        raise RuntimeError(f"{REF_LIBS[variant]} missing: run 'make -C oracle ref'")
    with tempfile.TemporaryDirectory() as d:
        icdir = os.path.join(d, "ic")
        write_npy_dir(ic, icdir)
        out_npz = os.path.join(d, "out.npz")
        envs = dict(os.environ)
        envs.update({k: repr(float(v)) for k, v in env.items()})
        cmd = [sys.executable, os.path.join(HERE, "_ref_runner.py"), REF_LIBS[variant], icdir,
               str(int(nsteps)), out_npz, ",".join(names)]
        subprocess.run(cmd, check=True, env=envs, timeout=timeout,
                       stdout=subprocess.DEVNULL)
        res = dict(np.load(out_npz))
    out = {"dts": res["dts"], "seconds": float(res["seconds"])}
    for k in names:
        out[k] = res[k].reshape(storage_shape(k, ic.nx, ic.ny))
    return out


def run_reference_replicas(ic, env: dict, nsteps: int, warmup: int, replicas: int, variant: str = "c0",
                           timeout: float = 1800.0):
    """``replicas`` independent processes of the compiled reference, each
    integrating ``warmup`` untimed then ``nsteps`` timed steps from ``ic``, all
    started together (one process per host core).  Returns the per-replica
    seconds of the timed steps."""
    import subprocess
    import sys
    from simplevofsolver_b200.workloads import write_npy_dir
    if not reference_available(variant):
        raise RuntimeError(f"{REF_LIBS[variant]} missing: run 'make -C oracle ref'")
    with tempfile.TemporaryDirectory() as d:
        icdir = os.path.join(d, "ic")
        write_npy_dir(ic, icdir)
        envs = dict(os.environ)
        envs.update({k: repr(float(v)) for k, v in env.items()})
        envs["OMP_NUM_THREADS"] = "1"
        procs = []
        for r in range(replicas):
            out_npz = os.path.join(d, f"out{r}.npz")
            cmd = [sys.executable, os.path.join(HERE, "_ref_runner.py"), REF_LIBS[variant], icdir,
                   str(int(nsteps)), out_npz, "", str(int(warmup))]
            procs.append((subprocess.Popen(cmd, env=envs, stdout=subprocess.DEVNULL), out_npz))
        secs = []
        for pr, out_npz in procs:
            pr.wait(timeout=timeout)
            if pr.returncode != 0:
                raise RuntimeError("reference replica failed")
            secs.append(float(np.load(out_npz)["seconds"]))
    return secs


def run_oracle3d_replicas(n: int, ndrops: int, radii, seed: int, nsteps: int, warmup: int, replicas: int,
                          timeout: float = 3600.0):
    """``replicas`` independent single-core processes of the 3D restatement on
    the seeded droplet field at n^3 (``_oracle3d_runner.py``), started
    together; returns the per-replica seconds of the ``nsteps`` timed steps."""
    import subprocess
    import sys
    with tempfile.TemporaryDirectory() as d:
        envs = dict(os.environ)
        envs["OMP_NUM_THREADS"] = "1"
        procs = []
        for r in range(replicas):
            out = os.path.join(d, f"o{r}.npz")
            cmd = [sys.executable, os.path.join(HERE, "_oracle3d_runner.py"), str(n), str(ndrops), repr(radii[0]),
                   repr(radii[1]), str(seed), str(nsteps), str(warmup), out]
            procs.append((subprocess.Popen(cmd, env=envs, stdout=subprocess.DEVNULL), out))
        secs = []
        for pr, out in procs:
            pr.wait(timeout=timeout)
            if pr.returncode != 0:
                raise RuntimeError("3D oracle replica failed")
            secs.append(float(np.load(out)["seconds"]))
    return secs
