"""CPU: the C-ABI library builds, loads, exports every symbol its header
declares, and fails loudly (no CPU fallback) where no GPU is usable."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vd_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "vd_tess_calculate" in syms and "vd_tess_create" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol():
    from vorothree_b200 import _lib
    L = _lib.load()
    for s in declared_symbols():
        assert hasattr(L, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_no_silent_cpu_path():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import vorothree_b200 as v
    with pytest.raises(v.VoronoidError):
        v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(2, 2, 2))


def test_wall_id_rejected_before_device():
    import vorothree_b200 as v
    with pytest.raises(ValueError):
        v.Wall(-999, v.SphereGeometry([0, 0, 0], 1.0))


def test_header_is_plain_c(tmp_path):
    """The header is what a C, Rust (bindgen) or Go (cgo) binding reads: it
    must compile as strict C99, and a C program must link every declared
    entry point against the library and call the host-only parser."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    from vorothree_b200 import _lib
    _lib.load()
    syms = declared_symbols()
    src = tmp_path / "abi.c"
    src.write_text(
        "#include <stdio.h>\n#include <string.h>\n#include \"voronoid_b200.h\"\n"
        "typedef void (*fn)(void);\n"
        "static const fn all[] = {" + ", ".join(f"(fn){s}" for s in syms) + "};\n"
        "int main(void) {\n"
        "  const char* text = \"0 1.5 2 3\\n\\n7 -4e-1\\n\";\n"
        "  double xyz[6];\n  size_t n = 0;\n"
        "  if (vd_parse_generators(text, strlen(text), xyz, 2, &n) != VD_OK || n != 2) return 1;\n"
        "  if (xyz[0] != 1.5 || xyz[2] != 3.0 || xyz[3] != -0.4 || xyz[5] != 0.0) return 2;\n"
        "  if (vd_parse_generators(\"0 \\xff\", 3, xyz, 2, &n) != VD_EINVAL) return 3;\n"
        "  printf(\"%u\\n\", (unsigned)(sizeof(all) / sizeof(all[0])));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "abi"
    libdir = os.path.join(ROOT, "vorothree_b200")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(exe), "-L", libdir, "-lvoronoid_b200", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stderr)
    assert int(r.stdout.strip()) == len(syms)


@pytest.mark.parametrize("bmin,bmax", [([0, 0, 0], [1, 0, 1]), ([0, 0, 0], [1, 1, -1]),
                                       ([0, 0, float("nan")], [1, 1, 1]), ([0, 0, 0], [1, float("inf"), 1])])
def test_degenerate_box_rejected_before_device(bmin, bmax):
    """A box with no positive finite extent on an axis is refused with
    VD_EINVAL before any device is touched (so also on a host without GPU)."""
    import numpy as np
    from vorothree_b200 import _lib
    L = _lib.load()
    mn = np.asarray(bmin, np.float64)
    mx = np.asarray(bmax, np.float64)
    h = ctypes.c_void_p()
    rc = L.vd_tess_create(mn.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                          mx.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2, 2, 2, ctypes.byref(h))
    assert rc == _lib.VD_EINVAL
    assert b"extent" in L.vd_last_error(None)
