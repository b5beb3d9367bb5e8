"""C ABI of libnwb: the library loads, exports every symbol include/nwb.h
declares, validates its arguments, and its box mesh builder reproduces the
reference Mesh arrays (checked against the oracle).  CPU only: no call here
launches device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from nekwave_b200 import DgSolver, Mesh, _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(nwb_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert "nwb_solver_create" in names and len(names) >= 20
    for n in sorted(names):
        assert hasattr(L, n), n
    assert set(names) <= set(_lib.SIGNATURES), sorted(set(names) - set(_lib.SIGNATURES))


def test_version_and_status_strings():
    L = _lib.lib()
    assert L.nwb_version() == 1
    assert L.nwb_status_string(_lib.NWB_EINVAL) == b"NWB_EINVAL"


@pytest.mark.parametrize("args", [
    (5, (4, 4, 4), (0, 0, 0), (1, 1, 1), (0, 0, 0)),
    (8, (3, 2, 2), (0, 0, 0), (1, 1, 1), (1, 1, 1)),
    (3, (2, 3, 4), (0, 0, 0), (2, 2, 1), (1, 0, 1)),
    (2, (1, 1, 1), (-1, -1, -1), (1, 1, 1), (0, 0, 0)),
    (10, (1, 2, 1), (0, 0, 0), (0.5, 2, 1), (0, 1, 0)),
])
def test_box_mesh_matches_reference_arrays(args):
    N, nel, lo, hi, per = args
    m = Mesh(N)
    m.createBoxMesh(*nel, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], *per)
    o = O.box_mesh(*args)
    for k in ("z", "w", "D", "w3", "x", "y", "zc", "jac", "met", "vmin", "vplus", "bc",
              "nx", "ny", "nz", "dA"):
        np.testing.assert_array_equal(m._arrays[k], getattr(o, k), err_msg=k)
    assert m.computeMinNodeDistance() == O.dxmin(o)


def test_box_mesh_rejects_bad_arguments():
    L = _lib.lib()
    h = C.c_void_p()
    for bad in [(1, 2, 2, 2), (11, 2, 2, 2), (4, 0, 2, 2)]:
        st = L.nwb_box_mesh_create(*bad, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0, C.byref(h))
        assert st == _lib.NWB_EINVAL
        assert L.nwb_last_error()
    st = L.nwb_box_mesh_create(4, 2, 2, 2, 1.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0, C.byref(h))
    assert st == _lib.NWB_EINVAL and b"empty" in L.nwb_last_error()


def test_solver_create_validates_before_touching_a_device():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.nwb_solver_create(None, 1.0, 0, C.byref(h)) == _lib.NWB_EINVAL
    m = Mesh(4)
    m.createBoxMesh(2, 2, 2)
    d = m.desc()
    d.N = 11
    assert L.nwb_solver_create(C.byref(d), 1.0, 0, C.byref(h)) == _lib.NWB_EINVAL
    d = m.desc()
    assert L.nwb_solver_create(C.byref(d), 1.0, 7, C.byref(h)) == _lib.NWB_EINVAL
    # face points out of canonical order are refused (nwb_mesh_desc contract)
    a = m._arrays
    saved = a["vmin"].copy()
    a["vmin"][[0, 1]] = a["vmin"][[1, 0]]
    d = m.desc()
    st = L.nwb_solver_create(C.byref(d), 1.0, 0, C.byref(h))
    a["vmin"][:] = saved
    assert st == _lib.NWB_EINVAL and b"vol_idx_minus" in L.nwb_last_error()


def test_dg_solver_mirror_requires_initialize():
    s = DgSolver()
    with pytest.raises(RuntimeError):
        s.step(0.1, 0.0)
    with pytest.raises(ValueError):
        DgSolver(precision="fp16")
