"""CPU tests of the C-ABI boundary: the built library loads and exports every
function include/sbdx.h declares; calls that need no GPU fail cleanly."""
import ctypes
import os
import re

import pytest

import sbdx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            names |= set(re.findall(r"\b(sbdx_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    for must in ("sbdx_ctx_create", "sbdx_set_integrals", "sbdx_set_strings", "sbdx_build_connectivity",
                 "sbdx_diag_terms", "sbdx_sigma", "sbdx_davidson", "sbdx_rdm", "sbdx_energy_backward"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = sbdx.load_library()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_null_context_is_an_argument_error():
    lib = sbdx.load_library()
    assert lib.sbdx_build_connectivity(None) == 1
    assert lib.sbdx_ctx_create(None, 0) == 1
    assert lib.sbdx_last_error(None) == b"null context"


def test_no_device_is_a_cuda_error_not_a_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = sbdx.load_library()
    h = ctypes.c_void_p()
    assert lib.sbdx_ctx_create(ctypes.byref(h), 0) == 2
