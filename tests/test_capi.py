"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/ptychotomo_b200.h declares, and validates arguments on the host
before touching a GPU.  No compute call is made here."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from ptychotomo_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ptychotomo_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pt_\w+)\s*\(", text, re.M)))


def test_library_is_built_and_loads():
    assert _lib.LIB_PATH.exists(), "run python -m ptychotomo_b200.build"
    lib = _lib.lib()
    assert b"sm_100a" in lib.pt_version()   # the library reports the one target it is built for


def test_every_header_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pt_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    unbound = [n for n in names if n not in _lib.SIGNATURES]
    assert not unbound, f"declared but not bound in _lib.SIGNATURES: {unbound}"


def test_argument_validation_happens_on_host():
    lib = _lib.lib()
    h = ctypes.c_void_p()
    assert lib.pt_radon_create(16, 4, 12, ctypes.byref(h)) == _lib.PT_ERR_ARG     # n not a multiple of 8
    assert "multiple of 8" in _lib.last_error()
    assert lib.pt_radon_create(0, 4, 16, ctypes.byref(h)) == _lib.PT_ERR_ARG      # no angles
    assert lib.pt_radon_create(16, 4, 16, None) == _lib.PT_ERR_ARG                # null handle slot
    assert lib.pt_radon_create(16, 4, 40, ctypes.byref(h)) == _lib.PT_ERR_UNSUPPORTED  # 3n not compiled
    assert lib.pt_radon_create_ex(16, 4, 16, 5, ctypes.byref(h)) == _lib.PT_ERR_ARG
    assert lib.pt_ptycho_create(1, 32, 32, 1, 4, 16, 32, 8, ctypes.byref(h)) == _lib.PT_ERR_UNSUPPORTED
    assert lib.pt_ptycho_create(1, 32, 32, 1, 4, 16, 16, 32, ctypes.byref(h)) == _lib.PT_ERR_ARG
    assert lib.pt_radon_fwd(None, None, None, None) == _lib.PT_ERR_ARG
    assert lib.pt_ptycho_adj(None, None, None, None) == _lib.PT_ERR_ARG
    assert lib.pt_radon_destroy(None) == _lib.PT_OK
    assert lib.pt_ptycho_destroy(None) == _lib.PT_OK


def test_python_errors_carry_the_library_message():
    from ptychotomo_b200 import PtychotomoArgError, radonusfft
    with pytest.raises(PtychotomoArgError, match="multiple of 8"):
        radonusfft(16, 4, 12)
