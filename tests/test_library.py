"""CPU tests of the C-ABI library: it builds for sm_100a, loads, and exports
every entry point the headers under include/ declare. No compute calls."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from mercuda_b200 import build as B
from mercuda_b200.backend import DROP_IN_SYMBOLS, EXTENSION_SYMBOLS, load_library

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = []
    for header in sorted((ROOT / "include").glob("*.h")):
        text = header.read_text()
        names += re.findall(r"^\s*(?:int|void|const\s+\w+\s*\*|double)\s+(mercury_\w+)\s*\(", text, re.M)
    return names


def test_headers_declare_the_reference_abi():
    names = declared_symbols()
    for sym in DROP_IN_SYMBOLS:
        assert sym in names
    assert len(DROP_IN_SYMBOLS) == 16


def test_library_builds_and_exports_every_declared_symbol():
    lib_path = B.build()
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mercury_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = load_library()
    for sym in DROP_IN_SYMBOLS + EXTENSION_SYMBOLS:
        assert hasattr(lib, sym)


def test_configure_rejects_unknown_algorithms():
    lib = load_library()
    assert lib.mercury_cuda_configure(5) != 0
    assert lib.mercury_cuda_configure(11) != 0
