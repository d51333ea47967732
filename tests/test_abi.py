"""The C ABI: the library builds for sm_100a here and exports every function
that include/*.h declares. No compute calls (no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(shkz_b200_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "shkz_b200_project_host" in names
    assert "shkz_b200_create" in names


def test_library_exports_every_declared_symbol():
    from shiokaze_b200 import build, native
    build.build()
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_only():
    from shiokaze_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_python_binding_lists_every_export():
    from shiokaze_b200 import native
    assert set(native.EXPORTS) == set(declared_functions())
