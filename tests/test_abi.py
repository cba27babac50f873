"""CPU tests of the C ABI: the library builds, loads without a GPU and exports
every function that include/*.h declares (no compute calls)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import PKG, ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(", src):
            name = m.group(1)
            line_start = src.rfind("\n", 0, m.start()) + 1
            line = src[line_start:m.end()]
            if line.lstrip().startswith("#") or name in ("if", "for", "while", "sizeof", "defined", "return"):
                continue
            # a declaration: a return type precedes the name on the same logical line
            if re.match(r"\s*(EPHMC_API\s+)?(const\s+)?(void|int|double|short|unsigned|char|fftw_plan)\b", line):
                names.add(name)
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    import importlib.util
    spec = importlib.util.spec_from_file_location("ephmc_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    path = mod.build()
    return ctypes.CDLL(path)


def test_header_declares_functions():
    names = declared_functions()
    assert "ephmc_eval" in names and "ephmc_ctx_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_status_strings_without_gpu(lib):
    lib.ephmc_status_string.restype = ctypes.c_char_p
    lib.ephmc_version.restype = ctypes.c_char_p
    assert lib.ephmc_status_string(0) == b"ok"
    assert b"sm_100a" in lib.ephmc_version()
