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
    assert ctypes.sizeof(_capi.SxProfileArrays) == 152


def test_struct_layouts_match_c_compiler(tmp_path):
    """Every struct of include/sxhmm.h: size and field offsets as a C compiler
    lays them out equal the ctypes mirror's."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"sx_opts": _capi.SxOpts, "sx_search_cfg": _capi.SxSearchCfg, "sx_hit": _capi.SxHit,
               "sx_domain": _capi.SxDomain, "sx_profile_info": _capi.SxProfileInfo,
               "sx_profile_arrays": _capi.SxProfileArrays, "sx_search_stats": _capi.SxSearchStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sxhmm.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])
