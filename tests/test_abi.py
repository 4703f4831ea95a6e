"""The C-ABI libraries load on the CPU and export every symbol the public headers declare."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(REPO, "include", h) for h in sorted(os.listdir(os.path.join(REPO, "include"))) if h.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"^\s*typedef[^;]*;", "", src, flags=re.M)  # function-pointer types are not exports
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            if m.group(1) not in ("if", "sizeof", "defined"):
                names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "wtd_steps" in names and "wtd_create" in names
    assert len(names) >= 25


@pytest.mark.parametrize("project", ["t2d_slda", "c2_slda2d", "c1_bdg1d"])
def test_library_exports_all_declared_symbols(project):
    from wslda_b200 import build
    path = build.build(project)
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"{project}: missing exports {missing}"


def test_info_without_gpu():
    from wslda_b200 import load_library
    lib = load_library("t3d_slda")
    d = (ctypes.c_int * 3)()
    n, cd, nh, f, cm = (ctypes.c_int() for _ in range(5))
    assert lib.wtd_info(d, ctypes.byref(n), ctypes.byref(cd), ctypes.byref(nh), ctypes.byref(f), ctypes.byref(cm)) == 0
    assert list(d) == [8, 6, 12] and n.value == 576 and cd.value == 3 and nh.value == 3 and f.value == 111 and cm.value == 1
    assert lib.wtd_error_string(-3).decode().startswith("lattice")
