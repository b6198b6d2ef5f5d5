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
