"""Pin the CPU oracle to the reference's own golden data.

* the HMMER 3.4 fixture: 2 profiles x 10 targets, hmmsearch --max, 20 domain
  rows; seq score / seq bias / domain score within 0.1 bits and exact
  hmm/ali/env coordinates (src/hmmer/search.rs:316-355);
* the known answers of the reference's unit tests (alphabet.rs:134-146,
  parse.rs:332-370, model.rs:364-393, dp.rs:916-955, pipeline.rs:599-616,
  search.rs:282-305).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O


def _fixture(golden):
    o = O.Oracle(path=os.path.join(golden, "hmmer34_pair.hmm"))
    fa = O.read_fasta(os.path.join(golden, "hmmer34_targets.faa"))
    t = O.TargetBatch([O.encode(s) for _, s in fa])
    rows = [l.split("\t") for l in open(os.path.join(golden, "hmmer34_expected.tsv")).read().splitlines()]
    return o, fa, t, rows


def test_hmmer34_parity(golden):
    o, fa, t, rows = _fixture(golden)
    hits, doms = o.search(t, O.make_cfg(cutoff="E", seq=10.0, dom=10.0, filters=False), nthreads=4)
    names = [n for n, _ in fa]
    n = 0
    for r in rows:
        tgt, q = r[0], r[1]
        hs = [h for h in hits if names[h.target_index] == tgt and o.names[h.profile_index] == q]
        assert hs, f"missing hit {tgt} {q}"
        h = hs[0]
        assert abs(h.score - float(r[2])) <= 0.1, (tgt, q, h.score, r[2])
        assert abs(h.bias - float(r[3])) <= 0.1, (tgt, q, h.bias, r[3])
        rep = [doms[h.dom_offset + k] for k in range(h.ndom) if doms[h.dom_offset + k].reported]
        d = rep[int(r[4]) - 1]
        assert abs(d.score - float(r[5])) <= 0.1, (tgt, q, d.score, r[5])
        coords = [d.hmm_from, d.hmm_to, d.ali_from, d.ali_to, d.env_from, d.env_to]
        assert coords == [int(x) for x in r[7:13]], (tgt, q, coords, r[7:13])
        n += 1
    assert n == 20


def test_alphabet_known_answers():
    assert list(O.encode("ACDEFGHIKLMNPQRSTVWY")) == list(range(20))
    assert list(O.encode("uo")) == [1, 8]
    assert list(O.encode("BJZX*")) == [20, 21, 22, 23, 24]
    assert list(O.encode("m k\n")) == [10, 8]
    assert list(O.encode("-._~!1")) == [24, 24, 24, 24, 24, 24]


def test_parse_known_answers(golden):
    tiny = open(os.path.join(golden, "tiny.hmm")).read()
    o = O.Oracle(text=tiny)
    assert o.n == 1 and o.names[0] == "tiny" and o.m[0] == 3
    cut, st = o.header(0)
    assert tuple(cut[0:2]) == (20.0, 18.5)  # GA
    assert math.isnan(cut[2])  # no TC
    assert tuple(cut[4:6]) == (10.0, 9.0)  # NC
    assert not np.isnan(st).any()  # calibrated
    two = tiny + tiny.replace("NAME  tiny", "NAME  tiny2")
    o2 = O.Oracle(text=two)
    assert o2.n == 2 and o2.names[1] == "tiny2"
    with pytest.raises(ValueError):
        O.Oracle(text=tiny.replace("ALPH  amino", "ALPH  DNA"))
    with pytest.raises(ValueError):
        O.Oracle(text=tiny.replace("0.02 4.5 4.5 0.6 0.8 0.6 0.8", "0.02 x 4.5 0.6 0.8 0.6 0.8"))


def test_model_known_answers():
    # flat model: background emissions -> zero match scores (model.rs:376-385)
    m = 10
    bg = [0.0787945, 0.0151600, 0.0535222, 0.0668298, 0.0397062, 0.0695071, 0.0229198, 0.0590092, 0.0594422,
          0.0963728, 0.0237718, 0.0414386, 0.0482904, 0.0395639, 0.0540978, 0.0683364, 0.0540687, 0.0673417,
          0.0114135, 0.0304133]
    from sxhmm.synth import write_hmm_text
    tr = [0.9, 0.05, 0.05, 0.5, 0.5, 0.5, 0.5]
    txt = write_hmm_text("flat", m, [bg] * m, [tr] * (m + 1))
    o = O.Oracle(text=txt)
    a = o.arrays(0)
    assert np.abs(a["msc"][:24, 1:]).max() < 1e-5
    assert np.isinf(a["msc"][24, 1])
    # occupancy-weighted entry normalises over the exits reachable (model.rs:364-374)
    s = sum(math.exp(a["t"][7][k]) * (m - k + 1) for k in range(1, m + 1))
    assert abs(s - 1.0) < 1e-4
    # null model formula (model.rs:387-393)
    p1 = 300.0 / 301.0
    want = 300.0 * math.log(p1) + math.log(1.0 - p1)
    assert abs(O.null_score(300) - want) < 1e-3


def test_dp_known_answers(golden):
    o = O.Oracle(path=os.path.join(golden, "tiny.hmm"))
    seq = O.encode("GGMKAGGGMKAGG")
    f = o.forward(0, seq)
    b = o.backward(0, seq)
    assert abs(f - b) < 1e-3
    dec = o.decode(0, seq)
    assert abs(dec["fwd"] - f) < 1e-4 and abs(dec["bwd"] - b) < 1e-3
    seq2 = O.encode("GGMKAGGGGGGMKAGG")
    assert o.viterbi(0, seq2) <= o.forward(0, seq2) + 1e-4
    tr = o.viterbi_trace(0, seq2)
    assert len(tr) == 2
    assert (tr[0][0], tr[0][1]) == (3, 5) and (tr[1][0], tr[1][1]) == (12, 14)
    assert (tr[0][2], tr[0][3]) == (1, 3)
    assert abs(O.logsum(0.0, 0.0) - math.log(2)) < 1e-6
    assert O.logsum(float("-inf"), -2.0) == -2.0
    assert O.logsum(float("-inf"), float("-inf")) == float("-inf")


def test_pipeline_known_answers(golden):
    assert abs(O.gumbel_surv(0.0, 0.0, 1.0) - (1.0 - math.exp(-1.0))) < 1e-12
    assert O.exp_logsurv(-5.0, 0.0, 0.7) == 0.0
    assert abs(O.exp_logsurv(10.0, 0.0, 0.7) + 7.0) < 1e-12
    o = O.Oracle(path=os.path.join(golden, "tiny.hmm"))
    t = O.TargetBatch([O.encode("GGGGGMKAGGGGGGGGGGGGGGGGGGGGMKAGGGGG")])
    hits, doms = o.search(t, O.make_cfg(cutoff="T", seq=-1e9, dom=-1e9, filters=False), nthreads=1)
    assert len(hits) == 1 and hits[0].ndom == 2 and hits[0].score > 0
    assert (doms[0].ali_from, doms[0].ali_to) == (6, 8)


def test_search_known_answers(golden):
    o = O.Oracle(path=os.path.join(golden, "tiny.hmm"))
    t = O.TargetBatch([O.encode("GGGGMKAGGGG"), O.encode("WWWWWWWWWWW")])
    hits, doms = o.search(t, O.make_cfg(cutoff="T", seq=0.0, dom=0.0, filters=False), nthreads=1)
    assert len(hits) == 1 and hits[0].target_index == 0 and doms[hits[0].dom_offset].reported
    with pytest.raises(ValueError, match="TC bit thresholds unavailable on model tiny"):
        o.search(O.TargetBatch([O.encode("MKA")]), O.make_cfg(cutoff="TC"))


def test_unit_expectations_file(golden):
    meta = json.load(open(os.path.join(golden, "unit_expectations.json")))
    import hashlib
    for f, h in meta["sha256"].items():
        assert hashlib.sha256(open(os.path.join(golden, f), "rb").read()).hexdigest() == h
