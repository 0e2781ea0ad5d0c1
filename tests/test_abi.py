"""CPU-only checks of the drop-in boundary: the C-ABI library loads and
exports every entry point that include/lsstag_b200.h declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(lsg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("lsg_create", "lsg_set_matrix_csr", "lsg_setup", "lsg_solve", "lsg_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from lsstag_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_options_match_reference_defaults():
    from lsstag_b200 import _lib
    o = _lib.default_options()
    assert o.method == _lib.METHOD_FGMRES and o.precond == _lib.PC_MG
    assert o.n_pre == 0 and o.n_post == 3          # base_task_description.h:41-42
    assert o.max_it == 200                          # base_task_description.h:44
    assert o.omega == pytest.approx(0.805)          # ls_stag_real_constants.h:62
    assert o.eps == pytest.approx(1e-5)             # ls_stag_real_constants.h:47
    assert o.zline_reference == 1


def test_python_module_fails_loudly_without_library(tmp_path, monkeypatch):
    from lsstag_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(FileNotFoundError):
        _lib.load()
