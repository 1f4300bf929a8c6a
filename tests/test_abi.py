"""The C ABI library (padeops_b200/_lib/libpado.so) without a GPU: it loads,
exports every function include/pado.h declares, and its host-side argument
checks return the reference's init codes and the library's error codes
before anything touches a device."""
import ctypes
import os
import re

import pytest

from padeops_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pado.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pado_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    assert os.path.exists(L.LIB_PATH), "libpado.so is not built (python -c 'import __graft_entry__ as g; g.build()')"
    return L.lib()


def test_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 30
    raw = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert not [n for n in names if n not in L.SIGNATURES], [n for n in names if n not in L.SIGNATURES]


def test_init_codes_without_device(lib):
    """Too-short lines give the reference's init status (cd06.F90:153-168,
    cd10.F90:219-309, cf90.F90:123-168); bad arguments give PADO_E_*."""
    h = ctypes.c_void_p()
    assert lib.pado_cd06_init(ctypes.byref(h), 5, 0.1, 1, 0, 0) == 3
    assert lib.pado_cd06_init(ctypes.byref(h), 7, 0.1, 0, 0, 0) == 2
    assert lib.pado_cd10_init(ctypes.byref(h), 7, 0.1, 1, 0, 0) == 2
    assert lib.pado_cd10_init(ctypes.byref(h), 7, 0.1, 0, 0, 0) == 2
    assert lib.pado_cf90_init(ctypes.byref(h), 9, 1) == 7
    assert h.value is None
    assert lib.pado_create(ctypes.byref(h), 3, 64, 0.1, 1, 0, 0) == L.E_ARG      # no such scheme
    assert lib.pado_create(ctypes.byref(h), 0, 0, 0.1, 1, 0, 0) == L.E_ARG       # n < 1
    assert lib.pado_create(ctypes.byref(h), 1, 64, 0.0, 1, 0, 0) == L.E_ARG      # dx = 0
    assert lib.pado_create(None, 1, 64, 0.1, 1, 0, 0) == L.E_NULL
    lib.pado_destroy(None)                                                       # no-op


def test_diagnostics(lib):
    for code in (L.OK, L.E_BC, L.E_NULL, L.E_ALIAS, L.E_UNSUPPORTED, L.E_ARG, L.E_CUDA, L.E_SIZE,
                 L.E_TIMEOUT, L.E_NOMEM, L.E_STATE):
        assert lib.pado_strerror(code).decode()
    assert re.search(r"\d+\.\d+", lib.pado_version().decode())
    assert lib.pado_launch_count() >= 0


def test_null_handles(lib):
    assert lib.pado_apply(None, 1, 1, None, None, 1, 1, 0, 0, None) == L.E_NULL
    assert lib.pado_dd1(None, None, None, 1, 1, 0, 0, None) == L.E_NULL
    assert lib.pado_apply_adjoint(None, 1, 1, None, None, 1, 1, 0, 0, None) == L.E_NULL
    assert lib.pado_batch_create(None, None, 0) == L.E_NULL
