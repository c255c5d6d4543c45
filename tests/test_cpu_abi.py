"""CPU checks of the C ABI: the shared library loads without a GPU and exports every function that
include/sphb200.h declares (no compute calls are made here)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sphb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sphb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "sphb_sim_step" in names and "sphb_compute_sfc_keys" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from sphexa_b200 import lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.skip("library not built")
    lib = L.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    from sphexa_b200 import lib as L
    assert set(declared_functions()) == set(L.EXPORTED)


def test_defaults_without_gpu():
    import ctypes as C
    from sphexa_b200 import lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.skip("library not built")
    p = L.Params()
    L.load().sphb_default_params(C.byref(p))
    assert (p.ng0, p.ngmax, p.bucket_focus, p.precision) == (100, 150, 64, 0)
    assert abs(p.gamma - 5.0 / 3.0) < 1e-15 and p.Kcour == 0.2 and p.Krho == 0.06
    assert L.load().sphb_sort_by_key_static_max() == 1 << 20
