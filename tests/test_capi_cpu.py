"""CPU-only checks of the C ABI: the library loads, exports every entry point that
include/schwinger_amg.h declares, and its host-only functions behave (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT

from amg_schwingermodel_b200 import _lib, read_parameters

HEADER = ROOT / "include" / "schwinger_amg.h"


def declared_functions(header: Path):
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(amg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions(HEADER)
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_default_params_are_the_reference_defaults():
    p = _lib.default_params()
    # src/variables.cpp:46-87, include/params.h:63-65, src/main.cpp:61-65,129
    assert (p.cycle, p.nu1, p.nu2, p.nit, p.sap_tv_iters) == (1, 0, 2, 0, 4)
    assert (p.sap_gmres_m, p.sap_gmres_restarts, p.sap_gmres_tol, p.sap_tol) == (5, 5, 1e-3, 1e-10)
    assert (p.kcycle_m, p.kcycle_restarts, p.kcycle_tol) == (5, 2, 0.1)
    assert (p.coarse_m, p.coarse_restarts, p.coarse_tol) == (20, 20, 0.1)
    assert (p.outer_m, p.outer_restarts, p.outer_tol) == (20, 50, 1e-10)


def test_read_parameters(tmp_path):
    f = tmp_path / "parameters.dat"
    f.write_text("0 8 8 20 4 4\n1 4 4 20 4 4\n2 2 2 20 2 2")
    assert read_parameters(str(f)) == [[0, 8, 8, 20, 4, 4], [1, 4, 4, 20, 4, 4], [2, 2, 2, 20, 2, 2]]
    bad = tmp_path / "bad.dat"
    bad.write_text("0 8 8 x 4 4\n")
    with pytest.raises(_lib.AmgError) as e:
        read_parameters(str(bad))
    assert e.value.status == _lib.AMG_ERR_INVALID
    with pytest.raises(_lib.AmgError):
        read_parameters(str(tmp_path / "missing.dat"))


def test_status_strings():
    L = _lib.lib()
    for s in (0, 1, -1, -2, -3, -4, -5, -6):
        assert L.amg_status_string(s)
    assert L.amg_version() >= 100


def test_bad_blocking_is_rejected_on_the_host():
    """Host-side validation fails before any device work (the reference would exit(1) or
    silently mis-index, include/params.h:21-24)."""
    L = _lib.lib()
    p = _lib.default_params()
    h = C.c_void_p()
    for rows in ([0, 3, 8, 10, 4, 4], [0, 8, 8, 10, 3, 4], [0, 8, 8, 10, 3, 3]):
        r = np.array(rows, dtype=np.int32)
        st = L.amg_create(C.byref(h), 64, 64, 2, r.ctypes.data_as(C.c_void_p), -0.1, C.byref(p), 0)
        assert st in (_lib.AMG_ERR_INVALID, _lib.AMG_ERR_UNSUPPORTED), st
    r = np.array([0, 8, 8, 10, 4, 4], dtype=np.int32)
    st = L.amg_create(C.byref(h), 64, 64, 7, r.ctypes.data_as(C.c_void_p), -0.1, C.byref(p), 0)
    assert st == _lib.AMG_ERR_INVALID


def test_header_constants_match_the_python_binding():
    """Every integer constant the header defines has the same value in _lib: the status codes,
    precision, cycle and preconditioner selectors by name, the profiling slots through
    _lib.PROF_SLOTS."""
    consts = dict(re.findall(r"^#define (AMG_[A-Z0-9_]+)\s+\(?(-?\d+)\)?", HEADER.read_text(), flags=re.M))
    assert "AMG_PRECOND_NONE" in consts and len(consts) >= 20
    prof = {k: int(consts.pop(k)) for k in list(consts) if k.startswith("AMG_PROF_")}
    assert prof.pop("AMG_PROF_SLOTS") == len(_lib.PROF_SLOTS)
    assert {k[len("AMG_PROF_"):].lower(): v for k, v in prof.items()} == _lib.PROF_SLOTS
    missing = [k for k in consts if not hasattr(_lib, k)]
    assert not missing, missing
    wrong = {k: (v, getattr(_lib, k)) for k, v in consts.items() if getattr(_lib, k) != int(v)}
    assert not wrong, wrong
