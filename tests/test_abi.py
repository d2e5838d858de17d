"""The C-ABI library loads and exports every symbol include/gf_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_api():
    names = _declared()
    assert "gf_pf_run" in names and "gf_kf_batch" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from gfb200 import _lib as L
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from gfb200 import _lib as L
    assert sorted(L.EXPORTED) == _declared()


def test_version_callable_without_gpu():
    from gfb200 import _lib as L
    assert L.load().gf_version() >= 100
