"""The C-ABI library loads and exports every symbol include/gf_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re

import pytest

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


def test_library_exports_every_diagnostic_symbol():
    src = open(os.path.join(ROOT, "include", "gf_b200_diag.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = sorted(set(re.findall(r"\b(gfx_[a-z0-9_]+)\s*\(", src)))
    assert names == ["gfx_umma_selftest", "gfx_wait_selftest"]
    from gfb200 import _lib as L
    lib = C.CDLL(L.LIB_PATH)
    assert all(hasattr(lib, n) for n in names)


def test_python_binding_covers_the_header():
    from gfb200 import _lib as L
    assert sorted(L.EXPORTED) == _declared()


def test_version_callable_without_gpu():
    from gfb200 import _lib as L
    assert L.load().gf_version() >= 100


STRUCTS = {  # C type in include/gf_b200.h -> ctypes mirror in gfb200._lib
    "gf_lg_model": "LGModelC", "gf_rb_model": "RBModelC", "gf_pf_config": "PFConfigC",
    "gf_pf_out": "PFOutC", "gf_kf_out": "KFOutC", "gf_kf_grad_out": "KFGradOutC",
    "gf_kf_backward_out": "KFBackOutC", "gf_csmc_config": "CsmcConfigC", "gf_csmc_out": "CsmcOutC",
    "gf_srv_config": "SrvConfigC", "gf_srv_request": "SrvRequestC", "gf_srv_result": "SrvResultC",
    "gf_srv_metrics": "SrvMetricsC",
}


def test_struct_layouts_match_header(tmp_path):
    """Every ABI struct's size and field offsets, as gcc lays them out from the
    header, equal the ctypes mirror's (a stale mirror would make the library read
    past the caller's struct)."""
    import ctypes
    import json
    import shutil
    import subprocess

    from gfb200 import _lib as L
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gf_b200.h"', "int main(void) {",
             '  printf("{");']
    first = True
    for cname, pyname in STRUCTS.items():
        fields = [f[0] for f in getattr(L, pyname)._fields_]
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"{cname}\\": [%zu", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf(",%zu", offsetof({cname}, {f}));')
        lines.append('  printf("]");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = json.loads(subprocess.check_output([str(exe)]).decode())
    for cname, pyname in STRUCTS.items():
        st = getattr(L, pyname)
        want = [ctypes.sizeof(st)] + [getattr(st, f[0]).offset for f in st._fields_]
        assert got[cname] == want, (cname, got[cname], want)
