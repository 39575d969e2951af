"""The C ABI library loads and exports exactly what include/amg_b200.h declares (no
compute calls: these run without a GPU)."""

import re
from pathlib import Path

import pytest

from amjax_b200 import _native as N

HEADER = Path(__file__).resolve().parents[1] / "include" / "amg_b200.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(amg_[a-z0-9_]+)\s*\(", text)))


def test_library_built():
    assert N.lib_path().exists(), "run __graft_entry__.build() first"


def test_every_declared_symbol_is_exported_and_bound():
    lib = N.load(require_cuda=False)
    names = declared()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, f"{name} declared in the header but not bound in _native.py"
    assert set(N.SIGNATURES) == set(names)


def test_version_and_error_string():
    lib = N.load(require_cuda=False)
    assert b"sm_100a" in lib.amg_version()
    assert lib.amg_last_error() == b""


def test_compute_entry_points_refuse_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    with pytest.raises(RuntimeError):
        N.load(require_cuda=True)
