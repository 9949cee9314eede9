"""The C-ABI library loads without a GPU and exports every entry point that
include/bsn.h declares (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bsn.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bsn_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    import build_lib
    path = build_lib.build()
    return ctypes.CDLL(path), path


def test_header_declares_entry_points():
    names = declared()
    assert "bsn_euler3d_step_f64" in names and "bsn_fmr3d_step_f64" in names
    assert len(names) >= 30


def test_every_declared_symbol_is_exported(lib):
    L, path = lib
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (bsn_[a-z0-9_]+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    for n in declared():
        getattr(L, n)   # resolvable through dlsym


def test_python_binding_covers_header():
    from bsn._lib import SIGNATURES
    assert sorted(SIGNATURES) == declared()


def test_every_public_api_function_is_exported():
    import ast
    import bsn.api as api
    tree = ast.parse(open(api.__file__).read())
    public = [n.name for n in tree.body
              if isinstance(n, (ast.FunctionDef, ast.ClassDef)) and not n.name.startswith("_")]
    assert [n for n in public if n not in api.__all__] == []


def test_host_orbit_entry_points_without_gpu(lib):
    # bsn_nbody_step / bsn_kepler_* are host FP64 code paths of the library
    import bsn._lib as B
    L = B.load()
    arr = (B.bsn_bh * 2)()
    arr[0] = B.bsn_bh((ctypes.c_double * 3)(0.5, 0, 0), (ctypes.c_double * 3)(0, 0.5, 0), 0.5, 1e-4, 1e6, 0.01)
    arr[1] = B.bsn_bh((ctypes.c_double * 3)(-0.5, 0, 0), (ctypes.c_double * 3)(0, -0.5, 0), 0.5, 1e-4, 1e6, 0.01)
    st = (ctypes.c_double * 13)()
    assert L.bsn_kepler_init(arr, (ctypes.c_double * 3)(0, 0, 0), None, -1.0, st) == 0
    assert abs(st[3] - 1.0) < 1e-12
    F = (ctypes.c_double * 6)()
    assert L.bsn_nbody_step(arr, 2, 1e-3, F) == 0
    # without a GPU, context creation reports a CUDA error instead of crashing
    rc = L.bsn_ctx_create(ctypes.byref(ctypes.c_void_p()), 0, None)
    assert rc in (0, B.BSN_ERR_CUDA)
