"""TEST INFRASTRUCTURE ONLY — ctypes wrapper around the CPU oracle.

The oracle is a C++ restatement of the reference Rust engine
(src/hmmer/*.rs of raw-lab/sentinel-x); see oracle/sx_oracle.hpp.  Only the
test-suite, the smoke check and bench.py's CPU-baseline leg use it, and only as
the checker: nothing in the product library imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

NCODE = 25


class OrCfg(C.Structure):
    _fields_ = [("cutoff_kind", C.c_int32), ("filters", C.c_int32), ("null2", C.c_int32), ("has_z", C.c_int32),
                ("seq", C.c_double), ("dom", C.c_double), ("f1", C.c_double), ("f2", C.c_double),
                ("f3", C.c_double), ("z", C.c_double)]


class OrHit(C.Structure):
    _fields_ = [("profile_index", C.c_int32), ("target_index", C.c_int32), ("score", C.c_float),
                ("bias", C.c_float), ("evalue", C.c_double), ("nexpected", C.c_float), ("ndom", C.c_int32),
                ("dom_offset", C.c_int32)]


class OrDom(C.Structure):
    _fields_ = [("score", C.c_float), ("bias", C.c_float), ("c_evalue", C.c_double), ("i_evalue", C.c_double),
                ("hmm_from", C.c_int32), ("hmm_to", C.c_int32), ("ali_from", C.c_int32), ("ali_to", C.c_int32),
                ("env_from", C.c_int32), ("env_to", C.c_int32), ("reported", C.c_int32), ("pad", C.c_int32)]


class OrStage(C.Structure):
    _fields_ = [("usc", C.c_float), ("filtersc", C.c_float), ("vsc", C.c_float), ("fwdsc", C.c_float),
                ("bcksc", C.c_float), ("nullsc", C.c_float), ("stage_reached", C.c_int32), ("pass_f1", C.c_int32),
                ("pass_bias", C.c_int32), ("pass_f2", C.c_int32), ("pass_f3", C.c_int32), ("is_hit", C.c_int32),
                ("bits", C.c_float), ("bias", C.c_float), ("ndom", C.c_int32), ("nregions", C.c_int32)]


CUTOFF = {"E": 0, "T": 1, "GA": 2, "NC": 3, "TC": 4}

_lib = None


def build():
    """Compile liboracle.so with oracle/Makefile (g++)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    P, I32, I64, F, D = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    u8 = C.POINTER(C.c_uint8)
    i64p = C.POINTER(C.c_int64)
    sig = {
        "or_last_error": (C.c_char_p, []),
        "or_load_text": (P, [C.c_char_p, I64, C.c_char_p]),
        "or_load_file": (P, [C.c_char_p]),
        "or_free": (None, [P]),
        "or_count": (I32, [P]),
        "or_m": (I32, [P, I32]),
        "or_name": (C.c_char_p, [P, I32]),
        "or_header": (None, [P, I32, fp, dp]),
        "or_profile_arrays": (None, [P, I32, fp, fp, fp, fp, fp, fp]),
        "or_encode": (I64, [C.c_char_p, I64, u8]),
        "or_msv": (F, [P, I32, u8, I64]),
        "or_viterbi": (F, [P, I32, u8, I64]),
        "or_forward": (F, [P, I32, u8, I64, fp]),
        "or_backward": (F, [P, I32, u8, I64, fp]),
        "or_bias": (F, [P, I32, u8, I64]),
        "or_null": (F, [I64]),
        "or_xsc": (None, [I64, I32, fp]),
        "or_gumbel_surv": (D, [D, D, D]),
        "or_exp_logsurv": (D, [D, D, D]),
        "or_logsum": (F, [F, F]),
        "or_score_pair": (None, [P, I32, u8, I64, C.POINTER(OrCfg), C.POINTER(OrStage)]),
        "or_search": (P, [P, I64, u8, i64p, i64p, C.POINTER(OrCfg), I32]),
        "or_results_nhits": (I64, [P]),
        "or_results_ndoms": (I64, [P]),
        "or_results_copy": (None, [P, C.POINTER(OrHit), C.POINTER(OrDom)]),
        "or_results_free": (None, [P]),
        "or_time_pairs": (None, [P, I64, u8, i64p, i64p, C.POINTER(OrCfg), I32, I64, I64, D, i64p, dp, dp, i64p]),
        "or_score_all": (None, [P, I64, u8, i64p, i64p, I32, fp, fp, fp]),
        "or_decode": (F, [P, I32, u8, I64, I64, I32, fp, fp, fp, fp, fp, fp]),
        "or_viterbi_trace": (I32, [P, I32, u8, I64, C.POINTER(C.c_int32), I32]),
        "or_forward_f64": (D, [P, I32, u8, I64, I32, I32, I64, D]),
        "or_expected_counts_f64": (D, [P, I32, u8, I64, I32, dp, dp, dp, dp, dp]),
        "or_posterior_f64": (D, [P, I32, u8, I64, I32, dp, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _u8(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def encode(seq):
    """Digitise a protein string (alphabet.rs:91-93) -> uint8 array."""
    b = seq.encode() if isinstance(seq, str) else bytes(seq)
    out = np.zeros(max(1, len(b)), dtype=np.uint8)
    n = lib().or_encode(b, len(b), _u8(out))
    return out[:n].copy()


def make_cfg(cutoff="E", seq=10.0, dom=10.0, filters=True, null2=True, f1=0.02, f2=1e-3, f3=1e-5, z=None):
    return OrCfg(CUTOFF[cutoff], int(filters), int(null2), int(z is not None), float(seq), float(dom), f1, f2, f3,
                 float(z) if z is not None else 0.0)


class TargetBatch:
    """Digitised targets packed as one byte array with offsets/lengths."""

    def __init__(self, dsqs):
        self.lens = np.array([len(d) for d in dsqs], dtype=np.int64)
        self.offs = np.zeros(len(dsqs), dtype=np.int64)
        if len(dsqs):
            self.offs[1:] = np.cumsum(self.lens)[:-1]
        self.seq = np.concatenate([np.asarray(d, dtype=np.uint8) for d in dsqs]) if len(dsqs) else np.zeros(1, np.uint8)
        if self.seq.size == 0:
            self.seq = np.zeros(1, np.uint8)
        self.n = len(dsqs)

    @classmethod
    def from_packed(cls, seq, offs, lens):
        t = cls.__new__(cls)
        t.seq = np.ascontiguousarray(seq, dtype=np.uint8)
        t.offs = np.ascontiguousarray(offs, dtype=np.int64)
        t.lens = np.ascontiguousarray(lens, dtype=np.int64)
        t.n = len(lens)
        return t

    def dsq(self, i):
        return self.seq[self.offs[i]:self.offs[i] + self.lens[i]]


class Oracle:
    """A set of configured profiles held by the oracle."""

    def __init__(self, text=None, path=None, source="<stream>"):
        L = lib()
        if path is not None:
            self.h = L.or_load_file(path.encode())
        else:
            b = text.encode() if isinstance(text, str) else text
            self.h = L.or_load_text(b, len(b), source.encode())
        if not self.h:
            raise ValueError(L.or_last_error().decode())
        self.n = L.or_count(self.h)
        self.m = [L.or_m(self.h, i) for i in range(self.n)]
        self.names = [L.or_name(self.h, i).decode() for i in range(self.n)]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_free(self.h)
            self.h = None

    def header(self, i):
        cut = np.zeros(6, np.float32)
        st = np.zeros(6, np.float64)
        lib().or_header(self.h, i, _f(cut), _d(st))
        return cut, st

    def arrays(self, i):
        m = self.m[i]
        w = m + 1
        msc = np.zeros(NCODE * w, np.float32)
        mo = np.zeros(NCODE * w, np.float32)
        t8 = np.zeros(8 * w, np.float32)
        p8 = np.zeros(8 * w, np.float32)
        tbm = np.zeros(1, np.float32)
        compo = np.zeros(20, np.float32)
        lib().or_profile_arrays(self.h, i, _f(msc), _f(mo), _f(t8), _f(p8), _f(tbm), _f(compo))
        return dict(msc=msc.reshape(NCODE, w), mo=mo.reshape(NCODE, w), t=t8.reshape(8, w), p=p8.reshape(8, w),
                    msv_tbm=float(tbm[0]), compo=compo)

    def msv(self, i, dsq):
        d = np.ascontiguousarray(dsq, np.uint8)
        return lib().or_msv(self.h, i, _u8(d), len(d))

    def viterbi(self, i, dsq):
        d = np.ascontiguousarray(dsq, np.uint8)
        return lib().or_viterbi(self.h, i, _u8(d), len(d))

    def forward(self, i, dsq, specials=False):
        d = np.ascontiguousarray(dsq, np.uint8)
        if specials:
            sp = np.zeros(5 * (len(d) + 1), np.float32)
            r = lib().or_forward(self.h, i, _u8(d), len(d), _f(sp))
            return r, sp.reshape(5, len(d) + 1)
        return lib().or_forward(self.h, i, _u8(d), len(d), None)

    def backward(self, i, dsq, specials=False):
        d = np.ascontiguousarray(dsq, np.uint8)
        if specials:
            sp = np.zeros(5 * (len(d) + 1), np.float32)
            r = lib().or_backward(self.h, i, _u8(d), len(d), _f(sp))
            return r, sp.reshape(5, len(d) + 1)
        return lib().or_backward(self.h, i, _u8(d), len(d), None)

    def bias(self, i, dsq):
        d = np.ascontiguousarray(dsq, np.uint8)
        return lib().or_bias(self.h, i, _u8(d), len(d))

    def score_pair(self, i, dsq, cfg=None):
        d = np.ascontiguousarray(dsq, np.uint8)
        st = OrStage()
        c = cfg or make_cfg()
        lib().or_score_pair(self.h, i, _u8(d), len(d), C.byref(c), C.byref(st))
        return st

    def search(self, targets, cfg=None, nthreads=None):
        """search_profiles over all (profile, target) pairs -> (hits, doms) numpy records."""
        c = cfg or make_cfg()
        nthreads = nthreads or os.cpu_count()
        r = lib().or_search(self.h, targets.n, _u8(targets.seq), _i64(targets.offs), _i64(targets.lens), C.byref(c),
                            nthreads)
        if not r:
            raise ValueError(lib().or_last_error().decode())
        nh = lib().or_results_nhits(r)
        nd = lib().or_results_ndoms(r)
        hits = (OrHit * max(nh, 1))()
        doms = (OrDom * max(nd, 1))()
        lib().or_results_copy(r, hits, doms)
        lib().or_results_free(r)
        return list(hits)[:nh], list(doms)[:nd]

    def time_pairs(self, targets, cfg=None, nthreads=None, start=0, max_pairs=None, time_limit=15.0):
        c = cfg or make_cfg()
        nthreads = nthreads or os.cpu_count()
        npairs = self.n * targets.n
        maxp = npairs if max_pairs is None else max_pairs
        done = C.c_int64()
        cells = C.c_double()
        secs = C.c_double()
        nh = C.c_int64()
        lib().or_time_pairs(self.h, targets.n, _u8(targets.seq), _i64(targets.offs), _i64(targets.lens), C.byref(c),
                            nthreads, start, maxp, time_limit, C.byref(done), C.byref(cells), C.byref(secs),
                            C.byref(nh))
        return dict(pairs=done.value, cells=cells.value, seconds=secs.value, hits=nh.value, threads=nthreads)

    def score_all(self, targets, nthreads=None):
        """msv, viterbi, forward of every profile x target -> three (P, T) arrays."""
        n = self.n * targets.n
        out = [np.zeros(max(n, 1), np.float32) for _ in range(3)]
        lib().or_score_all(self.h, targets.n, _u8(targets.seq), _i64(targets.offs), _i64(targets.lens),
                           nthreads or os.cpu_count(), _f(out[0]), _f(out[1]), _f(out[2]))
        return [o[:n].reshape(self.n, targets.n) for o in out]

    def decode(self, i, dsq, l_cfg=None, multihit=True):
        d = np.ascontiguousarray(dsq, np.uint8)
        L = len(d)
        m = self.m[i]
        pm = np.zeros((L + 1) * (m + 1), np.float32)
        pii = np.zeros_like(pm)
        pn = np.zeros(L + 1, np.float32)
        pj = np.zeros_like(pn)
        pc = np.zeros_like(pn)
        bsc = np.zeros(1, np.float32)
        f = lib().or_decode(self.h, i, _u8(d), L, L if l_cfg is None else l_cfg, int(multihit), _f(pm), _f(pii), _f(pn),
                            _f(pj), _f(pc), _f(bsc))
        return dict(fwd=f, bwd=float(bsc[0]), pm=pm.reshape(L + 1, m + 1), pi=pii.reshape(L + 1, m + 1), pn=pn, pj=pj,
                    pc=pc)

    def viterbi_trace(self, i, dsq):
        d = np.ascontiguousarray(dsq, np.uint8)
        out = np.zeros(4 * 64, np.int32)
        n = lib().or_viterbi_trace(self.h, i, _u8(d), len(d), out.ctypes.data_as(C.POINTER(C.c_int32)), 64)
        return [tuple(int(v) for v in out[4 * q:4 * q + 4]) for q in range(min(n, 64))]

    def forward_f64(self, i, dsq, multihit=True, kind=0, idx=0, delta=0.0):
        d = np.ascontiguousarray(dsq, np.uint8)
        return lib().or_forward_f64(self.h, i, _u8(d), len(d), int(multihit), kind, idx, delta)

    def expected_counts_f64(self, i, dsq, multihit=True):
        d = np.ascontiguousarray(dsq, np.uint8)
        w = self.m[i] + 1
        dm = np.zeros(NCODE * w)
        di = np.zeros(NCODE * w)
        dt = np.zeros(7 * w)
        db = np.zeros(w)
        bsc = np.zeros(1)
        z = lib().or_expected_counts_f64(self.h, i, _u8(d), len(d), int(multihit), _d(dm), _d(di), _d(dt), _d(db),
                                         _d(bsc))
        return dict(lnz=z, bsc=float(bsc[0]), d_msc=dm.reshape(NCODE, w), d_isc=di.reshape(NCODE, w),
                    d_t=dt.reshape(7, w), d_tbm=db)

    def posterior_f64(self, i, dsq, multihit=True):
        d = np.ascontiguousarray(dsq, np.uint8)
        L = len(d)
        w = self.m[i] + 1
        pm = np.zeros((L + 1) * w)
        pii = np.zeros_like(pm)
        z = lib().or_posterior_f64(self.h, i, _u8(d), L, int(multihit), _d(pm), _d(pii))
        return z, pm.reshape(L + 1, w), pii.reshape(L + 1, w)


def calibration_scorer(nthreads=None):
    """Calibration scorer (see sxhmm.synth.calibrate) backed by the oracle."""
    def score(profiles, seqs):
        from sxhmm import synth
        o = Oracle(text="".join(synth.profile_text(p, cutoffs=False) for p in profiles))
        return o.score_all(TargetBatch(seqs), nthreads)
    return score


def null_score(l):
    return lib().or_null(l)


def xsc(l, multihit=True):
    out = np.zeros(16, np.float32)
    lib().or_xsc(l, int(multihit), _f(out))
    return out


def gumbel_surv(x, mu, lam):
    return lib().or_gumbel_surv(x, mu, lam)


def exp_logsurv(x, tau, lam):
    return lib().or_exp_logsurv(x, tau, lam)


def logsum(a, b):
    return lib().or_logsum(a, b)


def read_fasta(path):
    out = []
    for line in open(path):
        line = line.rstrip("\n")
        if line.startswith(">"):
            out.append([line[1:].strip(), ""])
        elif out:
            out[-1][1] += line.strip()
    return [(a, b) for a, b in out]
