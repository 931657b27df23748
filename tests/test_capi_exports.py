"""The C-ABI library builds, loads and exports every symbol declared in include/*.h (CPU only:
no compute calls)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(gtsc_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "gtsc_encode" in names and "gtsc_decode" in names


def test_library_exports_every_declared_symbol(G):
    L = G.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_declares_every_signature(G):
    """ctypes would silently truncate 64-bit arguments of an undeclared function."""
    L = G.lib()
    undeclared = [n for n in declared_symbols()
                  if getattr(L, n).argtypes is None and n not in ("gtsc_last_error", "gtsc_version")]
    assert not undeclared, f"no argtypes for {undeclared}"


def test_version_and_sizes(G):
    assert G.lib().gtsc_version().startswith(b"gtsc")
    assert [G.dtype_size(d) for d in range(6)] == [1, 2, 4, 8, 4, 8]
    assert G.dtype_size(17) == 0


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import gputimeseriescompressionoptimizer_b200 as g
    monkeypatch.setattr(g, "_lib", None)
    monkeypatch.setattr(g, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        g.lib()
