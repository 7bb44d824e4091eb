"""GPU parity: the CUDA path (through the C ABI) against the oracle.

* stage scores (msv, viterbi, forward, backward): bit-identical to the oracle
  (which is pinned to the reference's fixtures); bias-filter score within 2 f32
  ulps (the device evaluates it with the device log for filtering only; the
  host recomputes it exactly before any decision is final);
* full searches: identical hit and domain sets, bit-identical scores and
  identical coordinates, on the HMMER 3.4 fixture (filters off), the unit-test
  known answers, edge-case targets and seeded synthetic workloads with filters
  on (so MSV/bias/Viterbi/Forward decisions are compared too).
"""
import numpy as np
import pytest

from oracle import oracle as O
import sxhmm
from _workloads import (edge_targets, fixture_targets, fixture_text, long_workload, small_config,
                        small_profiles_text, tiny_text)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = sxhmm.Engine()
    yield e
    e.close()


def _same(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return np.array_equal(a, b) or bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def _stage_check(engine, text, seqs):
    o = O.Oracle(text=text)
    ps = engine.load_text(text)
    ts = engine.targets([s for _, s in seqs])
    dsq = [O.encode(s) for _, s in seqs]
    pp, pt = np.meshgrid(np.arange(o.n), np.arange(len(seqs)), indexing="ij")
    pp, pt = pp.ravel(), pt.ravel()
    got = engine.score_pairs(ps, ts, pp, pt)
    want = {k: np.zeros(len(pp), np.float32) for k in got}
    for q, (i, j) in enumerate(zip(pp, pt)):
        d = dsq[j]
        if len(d) == 0:
            continue
        want["msv"][q] = o.msv(i, d)
        want["viterbi"][q] = o.viterbi(i, d)
        want["forward"][q] = o.forward(i, d)
        want["backward"][q] = o.backward(i, d)
        want["bias"][q] = o.bias(i, d)
    for k in ("msv", "viterbi", "forward", "backward"):
        bad = np.nonzero(~((got[k] == want[k]) | (np.isnan(got[k]) & np.isnan(want[k]))))[0]
        assert bad.size == 0, (k, [(int(pp[b]), int(pt[b]), got[k][b], want[k][b]) for b in bad[:5]])
    assert _ulps(got["bias"], want["bias"]).max() <= 2
    return got


def test_stage_scores_fixture(engine):
    _stage_check(engine, fixture_text(), fixture_targets())


def test_stage_scores_edges(engine):
    text = tiny_text() + small_profiles_text()
    _stage_check(engine, text, edge_targets() + fixture_targets()[:3])


def test_stage_scores_synthetic(engine):
    w = small_config(1, 0.004)
    seqs = [(f"t{i}", "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets[:60])]
    _stage_check(engine, w.hmm_text(), seqs)


def _hits_oracle(text, seqs, cfg):
    o = O.Oracle(text=text)
    t = O.TargetBatch([O.encode(s) for _, s in seqs])
    hits, doms = o.search(t, cfg)
    out = []
    for h in hits:
        ds = [(d.score, d.bias, d.hmm_from, d.hmm_to, d.ali_from, d.ali_to, d.env_from, d.env_to, bool(d.reported),
               d.i_evalue, d.c_evalue) for d in doms[h.dom_offset:h.dom_offset + h.ndom]]
        out.append((h.profile_index, h.target_index, h.score, h.bias, h.evalue, h.nexpected, ds))
    return out


def _hits_gpu(engine, text, seqs, cfg_kw, profiles=None):
    ps = profiles if profiles is not None else engine.load_text(text)
    targets = sxhmm.Targets(seqs)
    cutoff = {"E": sxhmm.Cutoff.evalue(cfg_kw.get("seq", 10.0), cfg_kw.get("dom", 10.0)),
              "T": sxhmm.Cutoff.bits(cfg_kw.get("seq", 0.0), cfg_kw.get("dom", 0.0)),
              "GA": sxhmm.Cutoff.gathering(), "NC": sxhmm.Cutoff.noise(), "TC": sxhmm.Cutoff.trusted()}[
        cfg_kw.get("cutoff", "E")]
    sc = sxhmm.SearchConfig(cutoff, sxhmm.PipelineConfig(filters=cfg_kw.get("filters", True)), cfg_kw.get("z"))
    hits = sxhmm.search_profiles(ps, targets, sc, engine)
    out = []
    for h in hits:
        ds = [(d.score, d.bias, d.hmm_from, d.hmm_to, d.ali_from, d.ali_to, d.env_from, d.env_to, d.reported,
               d.i_evalue, d.c_evalue) for d in h.domains]
        pi = [i["name"] for i in ps.info].index(h.profile)
        out.append((pi, h.target_index, h.score, h.bias, h.evalue, h.nexpected, ds))
    return out


def _assert_same_hits(a, b):
    assert len(a) == len(b), (len(a), len(b), [x[:2] for x in a], [x[:2] for x in b])
    for x, y in zip(a, b):
        assert x[:2] == y[:2]
        assert np.float32(x[2]) == np.float32(y[2]) and np.float32(x[3]) == np.float32(y[3]), (x[:4], y[:4])
        assert (x[4] == y[4]) or (np.isnan(x[4]) and np.isnan(y[4]))
        assert np.float32(x[5]) == np.float32(y[5])
        assert len(x[6]) == len(y[6])
        for d, e in zip(x[6], y[6]):
            assert d[:9] == tuple(e[:9]) or (np.float32(d[0]) == np.float32(e[0]) and d[2:9] == tuple(e[2:9])), (d, e)


def _cmp(engine, text, seqs, **kw):
    ocfg = O.make_cfg(cutoff=kw.get("cutoff", "E"), seq=kw.get("seq", 10.0 if kw.get("cutoff", "E") == "E" else 0.0),
                      dom=kw.get("dom", 10.0 if kw.get("cutoff", "E") == "E" else 0.0),
                      filters=kw.get("filters", True), z=kw.get("z"))
    a = _hits_oracle(text, seqs, ocfg)
    b = _hits_gpu(engine, text, seqs, kw)
    _assert_same_hits(a, b)
    return a, b


def test_search_hmmer34_fixture(engine):
    """hmmsearch --max on the HMMER 3.4 fixture: identical to the oracle and
    within 0.1 bits / exact coordinates of HMMER 3.4 (search.rs:316-355)."""
    seqs = fixture_targets()
    _, hits = _cmp(engine, fixture_text(), seqs, filters=False)
    import os
    from _workloads import GOLDEN
    rows = [l.split("\t") for l in open(os.path.join(GOLDEN, "hmmer34_expected.tsv")).read().splitlines()]
    names = [n for n, _ in seqs]
    pnames = ["FAM14", "FAM18"]
    for r in rows:
        h = [x for x in hits if names[x[1]] == r[0] and pnames[x[0]] == r[1]][0]
        assert abs(h[2] - float(r[2])) <= 0.1 and abs(h[3] - float(r[3])) <= 0.1
        rep = [d for d in h[6] if d[8]]
        d = rep[int(r[4]) - 1]
        assert abs(d[0] - float(r[5])) <= 0.1
        assert list(d[2:8]) == [int(v) for v in (r[7], r[8], r[9], r[10], r[11], r[12])]


def test_search_fixture_filters_on(engine):
    _cmp(engine, fixture_text(), fixture_targets(), filters=True)


def test_search_unit_known_answers(engine):
    a, b = _cmp(engine, tiny_text(), [("s", "GGGGGMKAGGGGGGGGGGGGGGGGGGGGMKAGGGGG")], cutoff="T", seq=-1e9, dom=-1e9,
                filters=False)
    assert len(b) == 1 and len(b[0][6]) == 2 and (b[0][6][0][4], b[0][6][0][5]) == (6, 8)
    a, b = _cmp(engine, tiny_text(), [("hit", "GGGGMKAGGGG"), ("miss", "WWWWWWWWWWW")], cutoff="T", seq=0.0, dom=0.0,
                filters=False)
    assert len(b) == 1 and b[0][1] == 0 and b[0][6][0][8]


def _decode(x):
    return "".join("ACDEFGHIKLMNPQRSTVWY"[c] for c in x)


def test_search_marker_set_gathering(engine):
    """Marker-set shape (BUSCO/EukCC-like, shrunk): markers of M 200-1500
    planted once in most genomes; one search per genome with the profiles'
    gathering cutoffs (Cutoff::Gathering), filters on."""
    w = small_config(2, 0.02)
    text = w.hmm_text()
    ps = engine.load_text(text)
    total = 0
    for g0, n in w.truth["genomes"]:
        seqs = [(w.target_ids[i], _decode(w.targets[i])) for i in range(g0, g0 + n)]
        a = _hits_oracle(text, seqs, O.make_cfg(cutoff="GA", seq=0.0, dom=0.0))
        b = _hits_gpu(engine, text, seqs, {"cutoff": "GA"}, profiles=ps)
        _assert_same_hits(a, b)
        total += len(b)
    assert total > 0


def test_search_viral_screen_shape(engine):
    """Viral-screen shape (shrunk): many profiles of M 30-800 against short
    targets with skewed residue frequencies, E-value cutoffs, filters on."""
    w = small_config(4, 0.002)
    seqs = [(w.target_ids[i], _decode(s)) for i, s in enumerate(w.targets)]
    _cmp(engine, w.hmm_text(), seqs, filters=True)
    _cmp(engine, w.hmm_text(), seqs[:60], filters=False)


def test_long_profiles(engine):
    """Profiles longer than the warp-chunked kernels' 2048 columns (the long
    kernels: one CTA per pair, rows in global scratch): stage scores
    bit-identical to the oracle, and searches with filters on and off give the
    oracle's hits, including an empty target."""
    text, seqs = long_workload()
    _stage_check(engine, text, [q for q in seqs if q[1]])
    _, b = _cmp(engine, text, seqs, filters=True)
    assert {(h[0], h[1]) for h in b} >= {(0, 5), (0, 6), (0, 7)}
    _cmp(engine, text, seqs, cutoff="T", seq=-1e9, dom=-1e9, filters=False)
    ps = engine.load_text(text)
    ts = engine.targets([q[1] for q in seqs if q[1]])
    with pytest.raises(sxhmm.HmmError, match="M > 2048"):
        engine.posterior_grad(ps, ts, np.array([0], np.int32), np.array([5], np.int32), 2100)
    # the plain engine and sx_search_many take the same long-profile pass
    plain = sxhmm.Engine(plain=True)
    try:
        _assert_same_hits(_hits_oracle(text, seqs, O.make_cfg()), _hits_gpu(plain, text, seqs, {}))
    finally:
        plain.close()
    sets = [engine.load_text(part + "//\n") for part in text.split("//\n") if part.strip()]
    cfg = sxhmm.SearchConfig().to_c()
    many = engine.search_many(sets, ts, cfg)
    for st, got in zip(sets, many):
        assert _raw(got) == _raw(engine.search(st, ts, cfg))
    assert sum(len(h) for h, _ in many) > 0


def test_shape_table_same_hits():
    """A tuner's shape table (sx_set_shape_table) changes only the kernel
    shapes: with every profile on the widest Viterbi shape, or on the tuned
    ones, the hits equal the oracle's; a shape too narrow for M is refused."""
    w = small_config(1, 0.01)
    seqs = [(w.target_ids[i], _decode(s)) for i, s in enumerate(w.targets)]
    e = sxhmm.Engine()
    try:
        shapes = e.shapes("viterbi")
        widest = max(range(len(shapes)), key=lambda i: shapes[i][0] * shapes[i][1])
        e.set_shape_table("viterbi", np.full(2049, widest, np.int32))
        assert e.shape_for("viterbi", 150) == widest
        _cmp(e, w.hmm_text(), seqs, filters=True)
        narrow = min(range(len(shapes)), key=lambda i: shapes[i][0] * shapes[i][1])
        with pytest.raises(sxhmm.HmmError, match="fewer than M"):
            e.set_shape_table("viterbi", np.full(2049, narrow, np.int32))
        e.set_shape_table("viterbi", None)
        _cmp(e, w.hmm_text(), seqs, filters=True)
    finally:
        e.close()


def test_empty_inputs(engine):
    """No profiles (an empty HMM text) or no targets: no hits and no error,
    as the reference's reader and search give."""
    assert _hits_gpu(engine, "", [("a", "MKAGG")], {}) == _hits_oracle("", [("a", "MKAGG")], O.make_cfg()) == []
    cfg = {"cutoff": "T", "seq": -1e9, "dom": -1e9, "filters": False}
    assert _hits_gpu(engine, tiny_text(), [], cfg) == []
    ps = engine.load_text(tiny_text())
    ts = engine.targets(["MKA"])
    got = engine.score_pairs(ps, ts, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert all(len(v) <= 1 for v in got.values())


def test_missing_cutoff_raises_like_reference(engine):
    ps = engine.load_text(tiny_text())
    with pytest.raises(sxhmm.HmmError, match="TC bit thresholds unavailable on model tiny"):
        sxhmm.search_profiles(ps, sxhmm.Targets([("s", "MKA")]), sxhmm.SearchConfig(sxhmm.Cutoff.trusted()), engine)


def _oracle_arrays(text):
    """Configured profiles as the oracle's arrays (an independent restatement
    of Hmm::configure), in the form sx_profiles_from_arrays takes."""
    o = O.Oracle(text=text)
    out = []
    for i in range(o.n):
        a = o.arrays(i)
        cut, st = o.header(i)
        out.append(dict(name=o.names[i], m=o.m[i], msc=a["msc"], mo=a["mo"], t=a["t"], p=a["p"], compo=a["compo"],
                        msv_tbm=a["msv_tbm"], ga=cut[0:2], tc=cut[2:4], nc=cut[4:6], msv=st[0:2], viterbi=st[2:4],
                        forward=st[4:6]))
    return out


def test_profiles_from_arrays_same_as_text(engine):
    """Profiles handed over as configured arrays (the input of
    search_profiles(&[Profile], ...)) search exactly like the same file parsed
    by the library: same header fields, stage scores and hits."""
    w = small_config(1, 0.01)
    text = w.hmm_text()
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    pa = engine.load_arrays(_oracle_arrays(text))
    pt = engine.load_text(text)
    assert all(i["acc"] is None and i["desc"] is None for i in pa.info)  # none were given
    for a, b in zip(pa.info, pt.info):
        for k in ("name", "m", "calibrated"):
            assert a[k] == b[k], k
        for k in ("ga", "tc", "nc", "msv", "viterbi", "forward"):
            assert np.array_equal(np.array(a[k]), np.array(b[k]), equal_nan=True), k
    ts = engine.targets([s for _, s in seqs[:40]])
    pp, pt_ = np.meshgrid(np.arange(len(pa)), np.arange(40), indexing="ij")
    sa = engine.score_pairs(pa, ts, pp.ravel(), pt_.ravel())
    sb = engine.score_pairs(pt, ts, pp.ravel(), pt_.ravel())
    for k in sa:
        assert _same(sa[k], sb[k]), k
    _assert_same_hits(_hits_gpu(engine, text, seqs, {}, profiles=pt), _hits_gpu(engine, text, seqs, {}, profiles=pa))
    with pytest.raises(sxhmm.HmmError, match="M must be at least 1"):
        bad = dict(_oracle_arrays(text)[0], m=0)
        bad.update(msc=np.zeros(25), mo=np.zeros(25), t=np.zeros(8), p=np.zeros(8))
        engine.load_arrays([bad])


def _raw(hits_doms):
    hits, doms = hits_doms
    out = []
    for h in hits:
        ds = doms[h.domain_offset:h.domain_offset + h.ndomains]
        out.append((h.profile_index, h.target_index, h.qlen, h.tlen, h.score, h.bias, h.evalue, h.nexpected,
                    [(d.score, d.bias, d.c_evalue, d.i_evalue, d.hmm_from, d.hmm_to, d.ali_from, d.ali_to,
                      d.env_from, d.env_to, d.reported) for d in ds]))
    return out


def _same_info(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        for k in x:
            if isinstance(x[k], tuple):
                assert np.array_equal(np.array(x[k]), np.array(y[k]), equal_nan=True), k
            else:
                assert x[k] == y[k], k


def _digital(engine, w):
    lens = np.array([len(x) for x in w.targets], np.int64)
    offs = np.zeros(len(lens), np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    return engine.targets_digital(np.concatenate(w.targets), offs, lens)


def test_search_many_equals_separate_searches(engine):
    """sx_search_many over several profile sets returns, per set, exactly
    what separate sx_search calls return (how BUSCO/CheckV batch their files)."""
    from sxhmm import synth
    w = small_config(1, 0.01)
    sets = [engine.load_text(synth.profile_text(p)) for p in w.profiles[:5]]
    sets.append(engine.load_text("".join(synth.profile_text(p) for p in w.profiles[5:9])))
    ts = _digital(engine, w)
    for cut in (sxhmm.Cutoff.evalue(10.0, 10.0), sxhmm.Cutoff.gathering()):
        cfg = sxhmm.SearchConfig(cut).to_c()
        many = engine.search_many(sets, ts, cfg)
        assert len(many) == len(sets)
        for s, got in zip(sets, many):
            assert _raw(got) == _raw(engine.search(s, ts, cfg))
        assert sum(len(h) for h, _ in many) > 0
    tiny = engine.load_text(tiny_text())
    with pytest.raises(sxhmm.HmmError, match="TC bit thresholds unavailable on model tiny"):
        engine.search_many([sets[0], tiny], ts, sxhmm.SearchConfig(sxhmm.Cutoff.trusted()).to_c())


def test_profile_cache_round_trip(engine, tmp_path):
    """A set written by sx_profiles_save and read by sx_profiles_load_binary
    searches exactly like the parsed file; damaged caches are refused."""
    w = small_config(1, 0.01)
    text = w.hmm_text()
    ps = engine.load_text(text)
    path = tmp_path / "lib.sxp"
    ps.save(str(path))
    pb = engine.load_binary(str(path))
    _same_info(pb.info, ps.info)
    ts = _digital(engine, w)
    cfg = sxhmm.SearchConfig().to_c()
    assert _raw(engine.search(pb, ts, cfg)) == _raw(engine.search(ps, ts, cfg))
    data = path.read_bytes()
    bad = bytearray(data)
    bad[len(bad) // 2] ^= 0x40
    (tmp_path / "flip.sxp").write_bytes(bytes(bad))
    with pytest.raises(sxhmm.HmmError, match="checksum mismatch"):
        engine.load_binary(str(tmp_path / "flip.sxp"))
    (tmp_path / "cut.sxp").write_bytes(data[: len(data) // 3])
    with pytest.raises(sxhmm.HmmError, match="checksum mismatch|bad magic"):
        engine.load_binary(str(tmp_path / "cut.sxp"))
    (tmp_path / "text.sxp").write_bytes(text.encode()[:4096])
    with pytest.raises(sxhmm.HmmError, match="bad magic"):
        engine.load_binary(str(tmp_path / "text.sxp"))
    with pytest.raises(sxhmm.HmmError):
        engine.load_binary(str(tmp_path / "missing.sxp"))


def test_digital_targets_validated(engine):
    """Digitised targets: a code above 24 ('*') is rejected with its position;
    the same residues as text and as codes give the same scores."""
    seqs = [("a", "MKTAYIAKQR"), ("b", "ACDEFGHIKLMNPQRSTVWY*XBZ")]
    codes = [O.encode(s) for _, s in seqs]
    lens = np.array([len(c) for c in codes], np.int64)
    offs = np.array([0, lens[0]], np.int64)
    flat = np.concatenate(codes).astype(np.uint8)
    ts = engine.targets_digital(flat, offs, lens)
    tt = engine.targets([s for _, s in seqs])
    ps = engine.load_text(tiny_text())
    pp, pt = np.zeros(2, np.int32), np.arange(2, dtype=np.int32)
    a = engine.score_pairs(ps, ts, pp, pt)
    b = engine.score_pairs(ps, tt, pp, pt)
    for k in a:
        assert _same(a[k], b[k]), k
    bad = flat.copy()
    bad[lens[0] + 3] = 25
    with pytest.raises(sxhmm.HmmError, match="residue code 25 out of range in target 1"):
        engine.targets_digital(bad, offs, lens)


def test_search_edges(engine):
    text = tiny_text() + small_profiles_text()
    _cmp(engine, text, edge_targets(), cutoff="T", seq=-1e9, dom=-1e9, filters=False)


@pytest.mark.parametrize("cutoff", ["E", "GA", "NC", "TC"])
def test_search_synthetic_config0(engine, cutoff):
    """The CPU-runnable configuration at full size: 1 profile of M = 100
    against 1,000 targets (L 100-500, 5% planted homologs), filters on."""
    w = small_config(0, 1.0)
    assert len(w.targets) == 1000 and w.profiles[0].m == 100
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    a, b = _cmp(engine, w.hmm_text(), seqs, cutoff=cutoff, filters=True)
    if cutoff == "E":  # every planted homolog is reported
        planted = {t for _, t in w.truth.get("homologs", [])}
        assert planted and planted <= {x[1] for x in b}


def test_search_synthetic_multiprofile(engine):
    w = small_config(1, 0.01)
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    _cmp(engine, w.hmm_text(), seqs, filters=True)
    st = engine.stats()
    assert st["pairs_in"][0] == len(w.profiles) * len(seqs)


def test_plain_engine_same_hits():
    """The plain one-pair-per-block kernels (SX_FLAG_PLAIN) give the same hits."""
    w = small_config(1, 0.01)
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    plain = sxhmm.Engine(plain=True)
    try:
        a = _hits_oracle(w.hmm_text(), seqs, O.make_cfg())
        b = _hits_gpu(plain, w.hmm_text(), seqs, {})
        _assert_same_hits(a, b)
    finally:
        plain.close()


def test_pipeline_blocks_same_hits():
    """Profile blocks whose host domain definition overlaps later blocks'
    device cascade (pipeline_blocks=3) give the oracle's hits, as one block does."""
    w = small_config(1, 0.01)
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    a = _hits_oracle(w.hmm_text(), seqs, O.make_cfg())
    for nb in (1, 3):
        e = sxhmm.Engine(pipeline_blocks=nb)
        try:
            _assert_same_hits(a, _hits_gpu(e, w.hmm_text(), seqs, {}))
            st = e.stats()
            assert st["pairs_in"][0] == len(w.profiles) * len(seqs)
            assert st["ms"][5] >= 0 and st["ms"][7] <= st["ms"][6]
        finally:
            e.close()


@pytest.mark.parametrize("where", ["device", "host"])
def test_envelope_rescoring_device_and_host(where):
    """Envelope rescoring (full-matrix Forward/Backward, posterior, null2,
    optimal-accuracy coordinates) forced onto the device or the host: both
    give the oracle's hits, domains and coordinates, filters on and off."""
    e = sxhmm.Engine(envelopes=where)
    try:
        _cmp(e, fixture_text(), fixture_targets(), filters=False)
        _cmp(e, fixture_text(), fixture_targets(), filters=True)
        w = small_config(0, 0.2)
        seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
        _cmp(e, w.hmm_text(), seqs, filters=True)
        w = small_config(1, 0.01)
        seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
        _cmp(e, w.hmm_text(), seqs, filters=True)
        _cmp(e, tiny_text() + small_profiles_text(), edge_targets(), cutoff="T", seq=-1e9, dom=-1e9, filters=False)
        st = e.stats()
        assert (st["pairs_out"][5] > 0) == (where == "device")
    finally:
        e.close()


@pytest.mark.parametrize("traces", ["device", "host"])
def test_stochastic_traces_device_and_host(traces):
    """Multi-domain regions of homolog-heavy targets (0-3 planted domains per
    target, M = 300): their 200-trace ensembles sampled on the device (region
    Forward matrix, traces, per-position null2 sums; clustering on the host)
    or on the host give the oracle's hits, domains and coordinates."""
    from sxhmm import synth
    w = synth.make_config(3, scale=1 / 8)
    seqs = [(w.target_ids[i], "".join("ACDEFGHIKLMNPQRSTVWY"[x] for x in s)) for i, s in enumerate(w.targets)]
    e = sxhmm.Engine(envelopes="device", traces=traces)
    try:
        _cmp(e, w.hmm_text(), seqs, cutoff="T", seq=0.0, dom=0.0, filters=False)
        st = e.stats()
        if traces == "device":
            assert st["pairs_out"][6] > 0 and st["pairs_in"][6] == st["pairs_out"][6], st
            assert st["cells"][6] > 0
        else:
            assert st["pairs_in"][6] == 0
    finally:
        e.close()


def test_forward_error_vs_fp64_logspace(engine):
    """FP32 odds-space Forward with per-row scaling (bit-identical to the
    reference) against an FP64 log-space Forward: within 0.01 bits."""
    rng = np.random.default_rng(3)
    for cfg, scale in ((0, 0.05), (1, 0.004), (3, 1 / 16)):
        w = small_config(cfg, scale) if cfg != 3 else __import__("sxhmm").synth.make_config(3, scale=scale)
        text = w.hmm_text()
        o = O.Oracle(text=text)
        ps = engine.load_text(text)
        lens = np.array([len(s) for s in w.targets], np.int64)
        offs = np.zeros(len(lens), np.int64)
        offs[1:] = np.cumsum(lens)[:-1]
        ts = engine.targets_digital(np.concatenate(w.targets), offs, lens)
        pairs = w.pairs or [(p, t) for p in range(len(w.profiles)) for t in range(len(w.targets))]
        pick = rng.choice(len(pairs), size=min(60, len(pairs)), replace=False)
        pp = np.array([pairs[q][0] for q in pick], np.int32)
        pt = np.array([pairs[q][1] for q in pick], np.int32)
        fwd = engine.score_pairs(ps, ts, pp, pt, stages=("forward",))["forward"]
        err = [abs(float(f) - o.forward_f64(int(a), w.targets[b])) / np.log(2) for f, a, b in zip(fwd, pp, pt)]
        assert max(err) < 0.01, (cfg, max(err))
