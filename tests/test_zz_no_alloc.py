"""The allocation-free Viterbi entry point (sx_score_viterbi_static).

It serves callers that must not allocate GPU memory during a call -- a host
program sharing the GPU with another runtime whose caching allocator holds
almost all device memory, or a latency-bound caller that cannot absorb the
device-wide synchronisation cudaMalloc/cudaFree may imply.  Its scratch is a
fixed device array inside the library.  Here it is called through the C ABI
and must return exactly what sx_score_pairs returns for Viterbi (the
reference's scores, bit for bit), on two calls in a row -- the second call
reuses the array the first one left behind.  The file is named so pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import sxhmm
from sxhmm import _capi
from _workloads import edge_targets, fixture_targets, fixture_text, long_workload, small_profiles_text, tiny_text

pytestmark = pytest.mark.gpu


def _static_scores(engine, ps, ts, pp, pt):
    lib = _capi.load_library()
    pp = np.ascontiguousarray(pp, np.int32)
    pt = np.ascontiguousarray(pt, np.int32)
    out = np.full(len(pp), np.nan, np.float32)
    rc = lib.sx_score_viterbi_static(engine.h, ps.h, ts.h, pp.ctypes.data_as(C.POINTER(C.c_int32)),
                                     pt.ctypes.data_as(C.POINTER(C.c_int32)), len(pp),
                                     out.ctypes.data_as(C.POINTER(C.c_float)))
    if rc != 0:
        raise sxhmm.HmmError(rc, lib.sx_last_error().decode())
    return out


def test_static_matches_score_pairs_twice():
    eng = sxhmm.Engine()
    try:
        text = fixture_text() + tiny_text() + small_profiles_text()
        seqs = [s for _, s in fixture_targets() + edge_targets()]
        ps = eng.load_text(text)
        ts = eng.targets(seqs)
        rng = np.random.default_rng(17)
        for call in range(2):
            n = 300 if call == 0 else 1000
            pp = rng.integers(0, ps.n, size=n).astype(np.int32)
            pt = rng.integers(0, len(seqs), size=n).astype(np.int32)
            want = eng.score_pairs(ps, ts, pp, pt, stages=("viterbi",))["viterbi"]
            got = _static_scores(eng, ps, ts, pp, pt)
            assert np.array_equal(got, want), (call, np.nonzero(got != want)[0][:5])
        with pytest.raises(sxhmm.HmmError, match="exceed the fixed limit"):
            _static_scores(eng, ps, ts, np.zeros(8193, np.int32), np.zeros(8193, np.int32))
        text_long, seqs_long = long_workload()
        pl = eng.load_text(text_long)
        tl = eng.targets([s for _, s in seqs_long if s])
        with pytest.raises(sxhmm.HmmError, match="M > 2048"):
            _static_scores(eng, pl, tl, np.zeros(1, np.int32), np.zeros(1, np.int32))
    finally:
        eng.close()
