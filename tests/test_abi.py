"""The C-ABI library loads without a GPU and exports every symbol include/steps_b200.h
declares; argument checks that precede any CUDA call answer with the documented codes."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "steps_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_api():
    names = declared()
    for must in ("sg_create", "sg_run", "sg_get_tet_count", "sg_set_comp_count", "sg_run_noalloc"):
        assert must in names


def test_library_exports_every_declared_symbol(steps_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", steps_lib._name], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    assert steps_lib.sg_version() == 1


def test_python_binding_covers_header(steps_lib):
    from steps_b200 import _lib

    bound = set(_lib.PROTOTYPES) | {"sg_last_error", "sg_version", "sg_run_noalloc"}
    assert set(declared()) <= bound


def test_null_handle_is_an_argument_error(steps_lib):
    t = C.c_double()
    steps_lib.sg_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    assert steps_lib.sg_get_time(None, C.byref(t)) == 1
    assert b"null solver handle" in steps_lib.sg_last_error()


def test_noalloc_size_limits_without_gpu(steps_lib):
    f = steps_lib.sg_run_noalloc
    f.argtypes = [C.c_int32, C.c_int32, C.c_int32] + [C.c_void_p] * 9 + [
        C.c_uint64, C.c_double, C.c_double, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    assert f(70000, 3, 0, 1, 1, 1, 1, 1, None, None, None, 1, 0, 0.0, 1.0, 0, None, None, None) == 1
    assert b"ntets" in steps_lib.sg_last_error()
    assert f(60000, 8, 0, 1, 1, 1, 1, 1, None, None, None, 1, 0, 0.0, 1.0, 0, None, None, None) == 1
    assert b"ntets * nspec" in steps_lib.sg_last_error()
    assert f(100, 3, 65, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0.0, 1.0, 0, None, None, None) == 1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import importlib

    from steps_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        _lib.load()
    importlib.reload(_lib)
