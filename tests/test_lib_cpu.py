"""The C-ABI library loads and exports every symbol declared in include/*.h (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import pytest

from dcs245_classical_sampling_b200 import _lib

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dcs_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_is_built_and_loads():
    lib = _lib.load()
    assert lib.dcs_abi_version() == 1


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert names <= set(_lib.SIGNATURES), names - set(_lib.SIGNATURES)


def test_struct_layouts_match():
    lib = _lib.load()
    for i, dt in enumerate(_lib.STRUCTS):
        assert lib.dcs_struct_size(i) == dt.itemsize


def test_argument_errors_without_gpu():
    lib = _lib.load()
    rc = lib.dcs_block_tail(None, 4, None, None, 1, None)
    assert rc == _lib.E_ARG
    assert b"invalid" in lib.dcs_last_error()
    with pytest.raises(_lib.DCSError):
        _lib.check(rc)
