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


def test_ctypes_structs_match_the_header(tmp_path):
    """Every argument struct of the C ABI has the same size and field offsets
    in the header (compiled here with the system C compiler) as in the
    Python binding."""
    import subprocess
    from shiokaze_b200 import native
    structs = {"shkz_b200_config": native.Config, "shkz_b200_project_args": native.ProjectArgs,
               "shkz_b200_result": native.Result, "shkz_b200_extend_args": native.ExtendArgs,
               "shkz_b200_splat_args": native.SplatArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "shkz_b200.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    include = os.path.join(ROOT, "include")
    subprocess.check_call(["gcc", "-I", include, str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)], text=True).split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_conv_entry_points_reject_before_device_work():
    """The convolution entry points refuse sizes and pointers they cannot take
    before they touch the device (these calls run without a GPU): a tensor-
    memory request above the SM's 512 columns (planes 8 with cout 128), and,
    for the no-allocation variant, activations or outputs off a 16-byte
    boundary."""
    import numpy as np
    from shiokaze_b200 import native
    L = native.load()
    buf = np.zeros(64, np.float32)
    p = buf.ctypes.data
    assert p % 16 == 0
    ERR_ARG, ERR_LIMIT = -1, -8
    # accumulators of 8 planes x 128 columns = 1024 > 512
    assert L.shkz_b200_conv3d(16, 32, 16, 16, 0, 128, 8, p, None, p, None, 1, p) == ERR_LIMIT
    assert L.shkz_b200_conv3d(16, 32, 16, 16, 0, 96, 8, p, None, p, None, 1, p) == ERR_LIMIT
    assert L.shkz_b200_conv3d_noalloc(16, 32, 16, 16, 0, 128, 8, p, None, p, None, 1, p, None) == ERR_LIMIT
    # misaligned in0, in1, out (16 bytes) and w (4 bytes)
    assert L.shkz_b200_conv3d_noalloc(16, 32, 16, 16, 0, 16, 8, p + 8, None, p, None, 1, p, None) == ERR_ARG
    assert L.shkz_b200_conv3d_noalloc(16, 32, 16, 16, 16, 16, 8, p, p + 4, p, None, 1, p, None) == ERR_ARG
    assert L.shkz_b200_conv3d_noalloc(16, 32, 16, 16, 0, 16, 8, p, None, p, None, 1, p + 2, None) == ERR_ARG
    assert L.shkz_b200_conv3d_noalloc(16, 32, 16, 16, 0, 16, 8, p, None, p + 2, None, 1, p, None) == ERR_ARG
    # sizes beyond the fixed scratch
    assert L.shkz_b200_conv3d_noalloc(16, 16, 16, 16, 0, 256, 4, p, None, p, None, 1, p, None) == ERR_LIMIT
    assert L.shkz_b200_conv3d_noalloc(16, 16, 16, 128, 16, 16, 8, p, p, p, None, 1, p, None) == ERR_LIMIT
