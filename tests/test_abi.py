"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; the Python host binds them all.  No compute call is
made here (that needs a GPU)."""
import ctypes
import glob
import os
import re

import pytest

import simplevofsolver_b200 as svof

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(svof(?:3d)?_[A-Za-z0-9_]+)\s*\(",
                             text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_abi():
    names = declared_functions()
    assert "svof_create" in names and "svof_integrate" in names
    assert len(names) >= 25


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = svof.lib()
    assert hasattr(lib, name), name


def test_python_host_binds_every_exported_entry():
    declared = set(declared_functions())
    assert set(svof.EXPORTS) <= declared
    assert set(svof.EXPORTS3D) <= declared
    assert {n for n in declared if n.startswith("svof3d_")} == set(svof.EXPORTS3D)


def test_every_declared_entry_has_argtypes():
    """the Python host declares the argument types of every C-ABI function
    (the two error-string getters take none)"""
    from simplevofsolver_b200.solver3d import lib3
    L = lib3()
    for name in declared_functions():
        if name in ("svof_last_error", "svof3d_last_error"):
            continue
        assert getattr(L, name).argtypes is not None, name


def test_create_fails_cleanly_without_device():
    """without a GPU, svof_create reports an error instead of crashing"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ic = svof.droplet2d(16, 16)
    with pytest.raises(svof.SvofError):
        svof.Solver(ic, svof.physical_params(svof.DROPLET2D_ENV))


REFERENCE_ENTRY_POINTS = [
    "fluid_init", "fluid_save", "fluid_decide_dt", "fluid_predict_field", "fluid_compute_potential_dft",
    "fluid_compute_potential_dct", "fluid_correct_velocity", "fluid_update_pressure",
    "fluid_update_boundaries_ux", "fluid_update_boundaries_uy", "fluid_update_boundaries_p",
    "fluid_update_boundaries_psi", "fluid_update_boundaries_t", "interface_init", "interface_save",
    "interface_compute_curvature_tensor", "interface_compute_force", "interface_update_vof",
    "interface_update_boundaries_vof", "linear_system_init", "linear_system_finalise", "integrate",
]


def test_reference_signature_header_matches_exports():
    """include/svof_reference_abi.h declares the reference's solver entry
    points (include/fluid_solver.h, interface_solver.h, linear_system.h,
    integrate.h) and the library exports every one of them"""
    text = open(os.path.join(ROOT, "include", "svof_reference_abi.h")).read()
    lib = svof.lib()
    for name in REFERENCE_ENTRY_POINTS:
        assert re.search(r"\bint\s+" + name + r"\s*\(", text), name
        assert hasattr(lib, name), name
