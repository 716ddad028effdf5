"""The C-ABI libraries load without a GPU and export every symbol their
headers declare (no compute calls are made here)."""
import ctypes
import re
from pathlib import Path

import pytest

from sod2d_b200 import build

ROOT = Path(__file__).resolve().parents[1]


def declared(header):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sod_(?:gpu|host)_\w+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("sod2d_host.h", "libsod2d_host.so"), ("sod2d_gpu.h", "libsod2d_gpu.so")])
def test_library_exports_header_symbols(header, lib):
    path = build.LIBDIR / lib
    if not path.exists():
        build.build_all()
    L = ctypes.CDLL(str(path))
    names = declared(header)
    assert names, header
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_declares_every_gpu_symbol():
    from sod2d_b200 import gpu
    assert sorted(gpu.SIGNATURES) == declared("sod2d_gpu.h")


def test_binding_argument_counts_match_header():
    """Each ctypes signature has as many arguments as the C declaration."""
    from sod2d_b200 import gpu
    text = (ROOT / "include" / "sod2d_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    for name, (_, args) in gpu.SIGNATURES.items():
        m = re.search(r"\b" + name + r"\s*\(([^)]*)\)", text)
        assert m, name
        params = [p for p in m.group(1).split(",") if p.strip() and p.strip() != "void"]
        assert len(params) == len(args), (name, len(params), len(args))
