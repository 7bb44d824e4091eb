"""ctypes binding of libsxhmm.so (include/sxhmm.h)."""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SX_OK, SX_EINVAL, SX_ECUTOFF, SX_ENOMEM, SX_ECUDA, SX_ETIMEOUT, SX_EIO = range(7)
SX_CUT_EVALUE, SX_CUT_BITS, SX_CUT_GA, SX_CUT_NC, SX_CUT_TC = range(5)
SX_FLAG_PLAIN = 1
SX_FLAG_ENV_DEVICE = 2
SX_FLAG_ENV_HOST = 4
SX_FLAG_TRACE_HOST = 8
SX_FLAG_TRACE_DEVICE = 16
SX_FLAG_NO_PRESCREEN = 32

# Every entry point declared in include/sxhmm.h, name -> (restype, argtypes).
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)


class SxOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("host_threads", C.c_int32), ("flags", C.c_uint32), ("pipeline_blocks", C.c_int32),
                ("batch_bytes", C.c_int64)]


class SxSearchCfg(C.Structure):
    _fields_ = [("cutoff_kind", C.c_int32), ("filters", C.c_int32), ("null2", C.c_int32), ("reserved", C.c_int32),
                ("seq_threshold", C.c_double), ("dom_threshold", C.c_double), ("f1", C.c_double), ("f2", C.c_double),
                ("f3", C.c_double), ("z", C.c_double)]


class SxHit(C.Structure):
    _fields_ = [("profile_index", C.c_int32), ("target_index", C.c_int32), ("qlen", C.c_int32), ("tlen", C.c_int32),
                ("score", C.c_float), ("bias", C.c_float), ("evalue", C.c_double), ("nexpected", C.c_float),
                ("ndomains", C.c_int32), ("domain_offset", C.c_int32), ("reserved", C.c_int32)]


class SxDomain(C.Structure):
    _fields_ = [("score", C.c_float), ("bias", C.c_float), ("c_evalue", C.c_double), ("i_evalue", C.c_double),
                ("hmm_from", C.c_int32), ("hmm_to", C.c_int32), ("ali_from", C.c_int32), ("ali_to", C.c_int32),
                ("env_from", C.c_int32), ("env_to", C.c_int32), ("reported", C.c_int32), ("reserved", C.c_int32)]


class SxProfileInfo(C.Structure):
    _fields_ = [("name", C.c_char_p), ("acc", C.c_char_p), ("desc", C.c_char_p), ("m", C.c_int32),
                ("calibrated", C.c_int32), ("ga", C.c_float * 2), ("tc", C.c_float * 2), ("nc", C.c_float * 2),
                ("msv", C.c_double * 2), ("viterbi", C.c_double * 2), ("forward", C.c_double * 2)]


class SxProfileArrays(C.Structure):
    _fields_ = [("name", C.c_char_p), ("acc", C.c_char_p), ("desc", C.c_char_p), ("m", C.c_int32),
                ("has_cutoffs", C.c_int32), ("msc", C.POINTER(C.c_float)), ("mo", C.POINTER(C.c_float)),
                ("t", C.POINTER(C.c_float)), ("p", C.POINTER(C.c_float)), ("compo", C.POINTER(C.c_float)),
                ("msv_tbm", C.c_float), ("ga", C.c_float * 2), ("tc", C.c_float * 2), ("nc", C.c_float * 2),
                ("has_stats", C.c_int32), ("msv", C.c_double * 2), ("viterbi", C.c_double * 2),
                ("forward", C.c_double * 2)]


class SxSearchStats(C.Structure):
    _fields_ = [("pairs_in", C.c_int64 * 8), ("pairs_out", C.c_int64 * 8), ("cells", C.c_double * 8),
                ("ms", C.c_double * 8), ("kernel_launches", C.c_int64), ("prescreen_pairs_in", C.c_int64),
                ("prescreen_pairs_out", C.c_int64), ("prescreen_cells", C.c_double), ("prescreen_ms", C.c_double),
                ("rescore_ms", C.c_double), ("vprescreen_pairs_in", C.c_int64),
                ("vprescreen_pairs_out", C.c_int64), ("vprescreen_cells", C.c_double), ("vprescreen_ms", C.c_double)]


_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_szp = C.POINTER(C.c_size_t)

SIGNATURES = {
    "sx_create": (C.c_int, [C.POINTER(SxOpts), _PP]),
    "sx_destroy": (None, [_P]),
    "sx_last_error": (C.c_char_p, []),
    "sx_profiles_load_file": (C.c_int, [_P, C.c_char_p, _PP]),
    "sx_profiles_load_text": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.c_char_p, _PP]),
    "sx_profiles_from_arrays": (C.c_int, [_P, C.POINTER(SxProfileArrays), C.c_size_t, _PP]),
    "sx_profiles_save": (C.c_int, [_P, C.c_char_p]),
    "sx_profiles_load_binary": (C.c_int, [_P, C.c_char_p, _PP]),
    "sx_profiles_count": (C.c_int32, [_P]),
    "sx_profiles_info": (C.c_int, [_P, C.c_int32, C.POINTER(SxProfileInfo)]),
    "sx_profiles_free": (None, [_P]),
    "sx_targets_create": (C.c_int, [_P, C.POINTER(C.c_char_p), C.POINTER(_u8p), _szp, C.c_size_t, _PP]),
    "sx_targets_create_digital": (C.c_int, [_P, _u8p, _i64p, _i64p, C.c_size_t, _PP]),
    "sx_targets_count": (C.c_int64, [_P]),
    "sx_targets_free": (None, [_P]),
    "sx_search": (C.c_int, [_P, _P, _P, C.POINTER(SxSearchCfg), _PP]),
    "sx_search_many": (C.c_int, [_P, C.POINTER(C.c_void_p), C.c_size_t, _P, C.POINTER(SxSearchCfg),
                                 C.POINTER(C.c_void_p)]),
    "sx_hits_count": (C.c_size_t, [_P]),
    "sx_hits_array": (C.POINTER(SxHit), [_P]),
    "sx_hits_domain_count": (C.c_size_t, [_P]),
    "sx_hits_domains": (C.POINTER(SxDomain), [_P]),
    "sx_hits_free": (None, [_P]),
    "sx_last_search_stats": (C.c_int, [_P, C.POINTER(SxSearchStats)]),
    "sx_shape_count": (C.c_int, [C.c_int]),
    "sx_shape_info": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sx_shape_for": (C.c_int, [_P, C.c_int, C.c_int32]),
    "sx_set_shape_table": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int32), C.c_size_t]),
    "sx_score_pairs": (C.c_int, [_P, _P, _P, _i32p, _i32p, C.c_size_t, _fp, _fp, _fp, _fp, _fp]),
    "sx_posterior_grad": (C.c_int, [_P, _P, _P, _i32p, _i32p, C.c_size_t, C.c_int32, _fp, _fp, _fp, _dp]),
    "sx_score_viterbi_static": (C.c_int, [_P, _P, _P, _i32p, _i32p, C.c_size_t, _fp]),
    "sx_score_prescreens": (C.c_int, [_P, _P, _P, _i32p, _i32p, C.c_size_t, _fp, _fp, _fp]),
}


class HmmError(RuntimeError):
    """An error returned by the engine (message from sx_last_error)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class LibraryMissing(RuntimeError):
    pass


def library_path():
    return os.environ.get("SXHMM_LIBRARY", os.path.join(HERE, "libsxhmm.so"))


_lib = None


def load_library():
    """Load libsxhmm.so; raise LibraryMissing if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise LibraryMissing(f"{path} not built: run `python sentinel-x_b200/build.py`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(rc):
    if rc != SX_OK:
        raise HmmError(rc, _lib.sx_last_error().decode(errors="replace"))


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Engine:
    """One engine per device (sx_create)."""

    def __init__(self, device=0, host_threads=0, plain=False, batch_bytes=0, pipeline_blocks=0, envelopes="auto",
                 traces="auto", prescreen=True):
        lib = load_library()
        flags = (SX_FLAG_PLAIN if plain else 0) | {"auto": 0, "device": SX_FLAG_ENV_DEVICE,
                                                    "host": SX_FLAG_ENV_HOST}[envelopes]
        flags |= 0 if prescreen else SX_FLAG_NO_PRESCREEN
        flags |= {"auto": 0, "device": SX_FLAG_TRACE_DEVICE, "host": SX_FLAG_TRACE_HOST}[traces]
        o = SxOpts(device, host_threads, flags, pipeline_blocks, batch_bytes)
        h = C.c_void_p()
        _check(lib.sx_create(C.byref(o), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib.sx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_text(self, text, source="<stream>"):
        return Profiles(self, text=text, source=source)

    def load_file(self, path):
        return Profiles(self, path=path)

    def load_arrays(self, profiles):
        """Configured profiles as arrays (sx_profiles_from_arrays): a list of
        dicts with name, m, msc [25, M+1], mo [25, M+1], t [8, M+1], p [8, M+1],
        compo [20], msv_tbm and optional acc, desc, ga/tc/nc, msv/viterbi/forward."""
        return Profiles(self, arrays=profiles)

    def targets(self, seqs, ids=None):
        return TargetSet(self, seqs=seqs, ids=ids)

    def targets_digital(self, seq, offs, lens):
        return TargetSet(self, digital=(seq, offs, lens))

    def search(self, profiles, targets, cfg):
        """Raw sx_search -> (hits structured array, domains structured array)."""
        out = C.c_void_p()
        _check(_lib.sx_search(self.h, profiles.h, targets.h, C.byref(cfg), C.byref(out)))
        return _take_hits(out)

    def search_many(self, sets, targets, cfg):
        """sx_search_many: one device search over several profile sets; a list
        with (hits, domains) per set, as search() would return for each."""
        n = len(sets)
        arr = (C.c_void_p * max(n, 1))(*[s.h for s in sets])
        outs = (C.c_void_p * max(n, 1))()
        _check(_lib.sx_search_many(self.h, arr, n, targets.h, C.byref(cfg), outs))
        return [_take_hits(C.c_void_p(outs[i])) for i in range(n)]

    def load_binary(self, path):
        """Profiles from a cache written by Profiles.save (sx_profiles_load_binary)."""
        return Profiles(self, binary=path)

    # kernel shapes, for tuners: kind "msv" or "viterbi"
    _KINDS = {"msv": 0, "viterbi": 1}

    def shapes(self, kind):
        """The compiled shapes of `kind` as (G, C, register transitions)."""
        k = self._KINDS[kind]
        out = []
        for i in range(_lib.sx_shape_count(k)):
            g, c, rt = C.c_int32(), C.c_int32(), C.c_int32()
            _check(_lib.sx_shape_info(k, i, C.byref(g), C.byref(c), C.byref(rt)))
            out.append((g.value, c.value, rt.value))
        return out

    def shape_for(self, kind, m):
        return _lib.sx_shape_for(self.h, self._KINDS[kind], int(m))

    def set_shape_table(self, kind, table):
        """Shape index per M = 0..2048 (-1 = the cost model), or None to
        restore the built-in table; applies to profile sets loaded afterwards."""
        if table is None:
            _check(_lib.sx_set_shape_table(self.h, self._KINDS[kind], None, 0))
            return
        t = np.ascontiguousarray(table, dtype=np.int32)
        _check(_lib.sx_set_shape_table(self.h, self._KINDS[kind], _ptr(t, C.c_int32), len(t)))

    def stats(self):
        s = SxSearchStats()
        _check(_lib.sx_last_search_stats(self.h, C.byref(s)))
        return {"pairs_in": list(s.pairs_in), "pairs_out": list(s.pairs_out), "cells": list(s.cells),
                "ms": list(s.ms), "kernel_launches": s.kernel_launches,
                "prescreen": {"pairs_in": s.prescreen_pairs_in, "pairs_out": s.prescreen_pairs_out,
                              "cells": s.prescreen_cells, "ms": s.prescreen_ms, "rescore_ms": s.rescore_ms},
                "vprescreen": {"pairs_in": s.vprescreen_pairs_in, "pairs_out": s.vprescreen_pairs_out,
                               "cells": s.vprescreen_cells, "ms": s.vprescreen_ms}}

    def score_pairs(self, profiles, targets, pp, pt, stages=("msv", "viterbi", "forward", "backward", "bias")):
        pp = np.ascontiguousarray(pp, dtype=np.int32)
        pt = np.ascontiguousarray(pt, dtype=np.int32)
        n = len(pp)
        out = {s: np.full(max(n, 1), np.nan, dtype=np.float32) for s in stages}

        def p(s):
            return _ptr(out[s], C.c_float) if s in out else None
        _check(_lib.sx_score_pairs(self.h, profiles.h, targets.h, _ptr(pp, C.c_int32), _ptr(pt, C.c_int32), n,
                                   p("msv"), p("viterbi"), p("forward"), p("backward"), p("bias")))
        return {s: v[:n] for s, v in out.items()}

    def score_prescreens(self, profiles, targets, pp, pt):
        """The conservative screens for explicit pairs (sx_score_prescreens):
        {"msv_bound": packed MSV pre-screen bound, "fwd_scan": F3 pre-screen
        Forward score, "vit_bound": packed Viterbi pre-screen bound}, float32
        arrays (nats)."""
        pp = np.ascontiguousarray(pp, dtype=np.int32)
        pt = np.ascontiguousarray(pt, dtype=np.int32)
        n = len(pp)
        mb = np.full(max(n, 1), np.nan, np.float32)
        fs = np.full(max(n, 1), np.nan, np.float32)
        vb = np.full(max(n, 1), np.nan, np.float32)
        _check(_lib.sx_score_prescreens(self.h, profiles.h, targets.h, _ptr(pp, C.c_int32), _ptr(pt, C.c_int32), n,
                                        _ptr(mb, C.c_float), _ptr(fs, C.c_float), _ptr(vb, C.c_float)))
        return {"msv_bound": mb[:n], "fwd_scan": fs[:n], "vit_bound": vb[:n]}

    def posterior_grad(self, profiles, targets, pp, pt, m, out=None):
        """lnZ and its gradients for each pair (sx_posterior_grad).  `out`:
        optional (lnz, d_msc, d_isc, d_tr) arrays to write into, of shapes (n,),
        (n, 25, m+1), (n, 25, m+1), (n, 8, m+1), float64 then float32,
        C-contiguous -- e.g. gradient buffers reused across calls, which spares
        the page faults of fresh memory."""
        pp = np.ascontiguousarray(pp, dtype=np.int32)
        pt = np.ascontiguousarray(pt, dtype=np.int32)
        n = len(pp)
        w = m + 1
        shapes = ((n,), (n, 25, w), (n, 25, w), (n, 8, w))
        dtypes = (np.float64, np.float32, np.float32, np.float32)
        if out is None:
            lnz, d_msc, d_isc, d_tr = (np.empty(sh, dt) for sh, dt in zip(shapes, dtypes))
        else:
            for a, sh, dt in zip(out, shapes, dtypes):
                if a.shape != sh or a.dtype != dt or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError(f"posterior_grad: out array must be a writeable C-contiguous {np.dtype(dt)} "
                                     f"array of shape {sh}")
            lnz, d_msc, d_isc, d_tr = out
        _check(_lib.sx_posterior_grad(self.h, profiles.h, targets.h, _ptr(pp, C.c_int32), _ptr(pt, C.c_int32), n, m,
                                      _ptr(d_msc, C.c_float), _ptr(d_isc, C.c_float), _ptr(d_tr, C.c_float),
                                      _ptr(lnz, C.c_double)))
        return lnz, d_msc, d_isc, d_tr


def _take_hits(out):
    try:
        nh = _lib.sx_hits_count(out)
        nd = _lib.sx_hits_domain_count(out)
        hits = [_copy(_lib.sx_hits_array(out)[i]) for i in range(nh)]
        doms = [_copy(_lib.sx_hits_domains(out)[i]) for i in range(nd)]
    finally:
        _lib.sx_hits_free(out)
    return hits, doms


def _copy(s):
    c = type(s)()
    C.pointer(c)[0] = s
    return c


class Profiles:
    """A configured profile set on the device (sx_profiles)."""

    def __init__(self, engine, text=None, path=None, source="<stream>", arrays=None, binary=None):
        self.engine = engine
        h = C.c_void_p()
        if binary is not None:
            _check(_lib.sx_profiles_load_binary(engine.h, os.fsencode(binary), C.byref(h)))
        elif arrays is not None:
            keep, recs = [], (SxProfileArrays * max(1, len(arrays)))()
            for i, a in enumerate(arrays):
                m = int(a["m"])
                buf = {k: np.ascontiguousarray(a[k], np.float32).ravel() for k in ("msc", "mo", "t", "p", "compo")}
                if buf["msc"].size != 25 * (m + 1) or buf["mo"].size != 25 * (m + 1) or buf["t"].size != 8 * (m + 1) \
                        or buf["p"].size != 8 * (m + 1) or buf["compo"].size != 20:
                    raise ValueError(f"profile {i}: array sizes do not match M = {m}")
                keep.append(buf)
                r = recs[i]
                r.name = a["name"].encode()
                r.acc = a["acc"].encode() if a.get("acc") else None
                r.desc = a["desc"].encode() if a.get("desc") else None
                r.m = m
                for k in ("msc", "mo", "t", "p", "compo"):
                    setattr(r, k, buf[k].ctypes.data_as(C.POINTER(C.c_float)))
                r.msv_tbm = float(a["msv_tbm"])
                r.has_cutoffs = 0
                for bit, k in enumerate(("ga", "tc", "nc")):
                    v = a.get(k)
                    if v is not None and not any(math.isnan(float(x)) for x in v):
                        r.has_cutoffs |= 1 << bit
                        setattr(r, k, (C.c_float * 2)(*[float(x) for x in v]))
                r.has_stats = 0
                for bit, k in enumerate(("msv", "viterbi", "forward")):
                    v = a.get(k)
                    if v is not None and not any(math.isnan(float(x)) for x in v):
                        r.has_stats |= 1 << bit
                        setattr(r, k, (C.c_double * 2)(*[float(x) for x in v]))
            _check(_lib.sx_profiles_from_arrays(engine.h, recs, len(arrays), C.byref(h)))
            del keep
        elif path is not None:
            _check(_lib.sx_profiles_load_file(engine.h, os.fsencode(path), C.byref(h)))
        else:
            b = text.encode() if isinstance(text, str) else bytes(text)
            _check(_lib.sx_profiles_load_text(engine.h, b, len(b), source.encode(), C.byref(h)))
        self.h = h
        self.n = _lib.sx_profiles_count(h)
        self.info = []
        for i in range(self.n):
            inf = SxProfileInfo()
            _check(_lib.sx_profiles_info(h, i, C.byref(inf)))
            self.info.append({
                "name": inf.name.decode(), "acc": inf.acc.decode() if inf.acc else None,
                "desc": inf.desc.decode() if inf.desc else None, "m": inf.m, "calibrated": bool(inf.calibrated),
                "ga": tuple(inf.ga), "tc": tuple(inf.tc), "nc": tuple(inf.nc),
                "msv": tuple(inf.msv), "viterbi": tuple(inf.viterbi), "forward": tuple(inf.forward)})

    def __len__(self):
        return self.n

    def save(self, path):
        """Write the configured set as a binary cache (sx_profiles_save)."""
        _check(_lib.sx_profiles_save(self.h, os.fsencode(path)))

    def close(self):
        if getattr(self, "h", None):
            _lib.sx_profiles_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TargetSet:
    """Digitised targets on the device (sx_targets)."""

    def __init__(self, engine, seqs=None, ids=None, digital=None):
        self.engine = engine
        h = C.c_void_p()
        if digital is not None:
            seq, offs, lens = digital
            seq = np.ascontiguousarray(seq, dtype=np.uint8)
            offs = np.ascontiguousarray(offs, dtype=np.int64)
            lens = np.ascontiguousarray(lens, dtype=np.int64)
            _check(_lib.sx_targets_create_digital(engine.h, _ptr(seq, C.c_uint8), _ptr(offs, C.c_int64),
                                                  _ptr(lens, C.c_int64), len(lens), C.byref(h)))
            self.n = len(lens)
        else:
            bs = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
            n = len(bs)
            arr = (_u8p * max(n, 1))()
            keep = []
            for i, b in enumerate(bs):
                buf = C.create_string_buffer(b, len(b) + 1)
                keep.append(buf)
                arr[i] = C.cast(buf, _u8p)
            lens = (C.c_size_t * max(n, 1))(*[len(b) for b in bs])
            idarr = None
            if ids is not None:
                idarr = (C.c_char_p * max(n, 1))(*[str(x).encode() for x in ids])
            _check(_lib.sx_targets_create(engine.h, idarr, arr, lens, n, C.byref(h)))
            self.n = n
        self.h = h

    def __len__(self):
        return self.n

    def close(self):
        if getattr(self, "h", None):
            _lib.sx_targets_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def search_cfg(cutoff_kind=SX_CUT_EVALUE, seq=10.0, dom=10.0, filters=True, null2=True, f1=0.02, f2=1e-3, f3=1e-5,
               z=None):
    return SxSearchCfg(cutoff_kind, int(filters), int(null2), 0, float(seq), float(dom), f1, f2, f3,
                       math.nan if z is None else float(z))
