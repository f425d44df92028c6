"""The C-ABI library loads without a GPU and exports every entry point that
include/fsb200.h declares (no compute calls here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "fsb200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from flowsolversourcecode_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header():
    from flowsolversourcecode_b200 import _lib as L
    assert set(_declared()) <= set(L.PROTOTYPES)


def test_struct_layout_matches_header():
    # the ctypes mirror of fs_case must have the C size (compiled probe)
    import subprocess, tempfile
    from flowsolversourcecode_b200 import _lib as L
    src = '#include "fsb200.h"\n#include <stdio.h>\nint main(){printf("%zu %zu %zu\\n", sizeof(fs_case), sizeof(fs_mesh_in), sizeof(fs_residuals));return 0;}\n'
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "p")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        out = subprocess.check_output([exe]).decode().split()
    assert int(out[0]) == ctypes.sizeof(L.FsCase)
    assert int(out[1]) == ctypes.sizeof(L.FsMeshIn)
    assert int(out[2]) == ctypes.sizeof(L.FsResiduals)
