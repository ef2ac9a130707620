"""The C-ABI library loads and exports every entry point the public headers
declare (no GPU needed; no compute calls are made)."""
import ctypes
import os
import re

import pytest

import mass_hd_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for f in sorted(os.listdir(INCLUDE)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(mass_(?:lb|sg)_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "mass_lb_create" in names and "mass_lb_step" in names
    assert len(names) >= 15


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = ctypes.CDLL(M.library_path())
    assert hasattr(lib, name), name


def test_abi_version_and_names():
    lib = M.load_library()
    assert lib.mass_lb_abi_version() == 1
    assert lib.mass_lb_field_name(0) == b"ff"
    assert lib.mass_lb_field_name(26) == b"sigma_active_yx"
    assert lib.mass_lb_field_name(99) is None
    assert [lib.mass_lb_field_name(i).decode() for i in range(len(M.FIELDS))] == list(M.FIELDS)
    assert lib.mass_lb_field_name(len(M.FIELDS)) is None
    assert lib.mass_lb_field_name(31) == b"m" and lib.mass_lb_field_name(32) == b"chi"


def test_create_rejects_bad_arguments_without_device():
    lib = M.load_library()
    h = ctypes.c_void_p()
    p = M.make_params(0, {})
    assert lib.mass_lb_create(None, 8, 8, 0, 0, ctypes.byref(h)) == -1
    assert lib.mass_lb_create(ctypes.byref(p), 0, 8, 0, 0, ctypes.byref(h)) == -1
    assert lib.mass_lb_create(ctypes.byref(p), 8, 8, 0, 7, ctypes.byref(h)) == -1
    p.npc = 0
    assert lib.mass_lb_create(ctypes.byref(p), 8, 8, 0, 0, ctypes.byref(h)) == -1


def test_nematic_rejects_thermal_noise():
    with pytest.raises(M.MassLBError):
        M.make_params(M.NEMATIC, {"Q_kBT": 0.1})


def test_ensemble_create_rejects_bad_arguments_without_device():
    lib = M.load_library()
    h = ctypes.c_void_p()
    P = M.lb.Params
    lx = (ctypes.c_uint * 2)(64, 64)
    ly = (ctypes.c_uint * 2)(64, 64)
    two = (P * 2)(M.make_params(0, {}), M.make_params(0, {}))
    assert lib.mass_lb_ensemble_create(0, two, lx, ly, ctypes.byref(h)) == -1
    assert lib.mass_lb_ensemble_create(2, None, lx, ly, ctypes.byref(h)) == -1
    assert lib.mass_lb_ensemble_create(193, two, lx, ly, ctypes.byref(h)) == -1
    mixed = (P * 2)(M.make_params(0, {}), M.make_params(1, {}))
    assert lib.mass_lb_ensemble_create(2, mixed, lx, ly, ctypes.byref(h)) == -1
    npc2 = (P * 2)(M.make_params(0, {"npc": 2}), M.make_params(0, {"npc": 2}))
    assert lib.mass_lb_ensemble_create(2, npc2, lx, ly, ctypes.byref(h)) == -4
    bad_ly = (ctypes.c_uint * 2)(64, 62)
    assert lib.mass_lb_ensemble_create(2, two, lx, bad_ly, ctypes.byref(h)) == -4
    assert h.value is None
    assert lib.mass_lb_ensemble_size(None) == 0
    assert lib.mass_lb_ensemble_run(None, 0) is None
    assert lib.mass_lb_ensemble_step(None, 1) == -1
