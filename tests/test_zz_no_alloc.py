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
        # no pairs: OK, and the output array is not touched
        lib = _capi.load_library()
        one = np.zeros(1, np.int32)
        out0 = np.full(4, np.nan, np.float32)
        assert lib.sx_score_viterbi_static(eng.h, ps.h, ts.h, one.ctypes.data_as(C.POINTER(C.c_int32)),
                                           one.ctypes.data_as(C.POINTER(C.c_int32)), 0,
                                           out0.ctypes.data_as(C.POINTER(C.c_float))) == 0
        assert np.isnan(out0).all()
        # exactly the limit
        pp = rng.integers(0, ps.n, size=8192).astype(np.int32)
        pt = rng.integers(0, len(seqs), size=8192).astype(np.int32)
        want = eng.score_pairs(ps, ts, pp, pt, stages=("viterbi",))["viterbi"]
        assert np.array_equal(_static_scores(eng, ps, ts, pp, pt), want)
        with pytest.raises(sxhmm.HmmError, match="exceed the fixed limit"):
            _static_scores(eng, ps, ts, np.zeros(8193, np.int32), np.zeros(8193, np.int32))
        text_long, seqs_long = long_workload()
        pl = eng.load_text(text_long)
        tl = eng.targets([s for _, s in seqs_long if s])
        with pytest.raises(sxhmm.HmmError, match="M > 2048"):
            _static_scores(eng, pl, tl, np.zeros(1, np.int32), np.zeros(1, np.int32))
    finally:
        eng.close()


def test_static_against_oracle_and_second_engine():
    """The static path's Viterbi scores equal the oracle's (the reference's
    f32 values) directly; a second engine on the same device, calling after
    the first engine's calls, reads back its own results from the shared
    array; handles of another engine are refused before anything launches."""
    from oracle import oracle as O
    text = fixture_text() + tiny_text() + small_profiles_text()
    seqs = [s for _, s in fixture_targets() + edge_targets()]
    o = O.Oracle(text=text)
    dsq = [O.encode(s) for s in seqs]
    rng = np.random.default_rng(23)
    e1, e2 = sxhmm.Engine(), sxhmm.Engine()
    try:
        p1, t1 = e1.load_text(text), e1.targets(seqs)
        p2, t2 = e2.load_text(text), e2.targets(seqs)
        pp = rng.integers(0, p1.n, size=400).astype(np.int32)
        pt = rng.integers(0, len(seqs), size=400).astype(np.int32)
        want = np.array([o.viterbi(int(i), dsq[j]) if len(dsq[j]) else np.nan for i, j in zip(pp, pt)], np.float32)
        got1 = _static_scores(e1, p1, t1, pp, pt)
        ok = (got1 == want) | (np.isnan(want) & np.isnan(got1))
        assert ok.all(), [(int(pp[q]), int(pt[q]), got1[q], want[q]) for q in np.nonzero(~ok)[0][:5]]
        pp2, pt2 = pp[::-1].copy(), pt[::-1].copy()
        got2 = _static_scores(e2, p2, t2, pp2, pt2)
        assert np.array_equal(got2, got1[::-1], equal_nan=True)
        with pytest.raises(sxhmm.HmmError, match="belong to another engine"):
            _static_scores(e1, p2, t1, pp[:4], pt[:4])
        with pytest.raises(sxhmm.HmmError, match="belong to another engine"):
            _static_scores(e1, p1, t2, pp[:4], pt[:4])
        with pytest.raises(sxhmm.HmmError, match="belong to another engine"):
            e1.score_pairs(p2, t1, pp[:4], pt[:4])
    finally:
        e1.close()
        e2.close()
