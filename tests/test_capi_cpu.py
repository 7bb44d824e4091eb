"""CPU-side checks of the product library: it is built, loads, exports every
entry point include/sxhmm.h declares, and fails cleanly (no crash) without a
GPU.  No compute call runs here."""
import ctypes
import os
import re

import pytest

import sxhmm
from sxhmm import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sxhmm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sx_[a-z_0-9]+)\s*\(", text)))


def test_header_lists_entry_points():
    syms = declared_symbols()
    assert "sx_search" in syms and "sx_create" in syms and "sx_posterior_grad" in syms
    assert set(syms) == set(_capi.SIGNATURES), set(syms) ^ set(_capi.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _capi.load_library()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    # and through the raw loader, independent of the binding
    raw = ctypes.CDLL(_capi.library_path())
    for s in declared_symbols():
        getattr(raw, s)


def test_no_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sxhmm.HmmError):
        sxhmm.Engine()
    assert sxhmm.load_library().sx_last_error()


def test_struct_sizes_match_header():
    assert ctypes.sizeof(_capi.SxHit) == 48
    assert ctypes.sizeof(_capi.SxDomain) == 56
    assert ctypes.sizeof(_capi.SxSearchCfg) == 64
    assert ctypes.sizeof(_capi.SxOpts) == 24
