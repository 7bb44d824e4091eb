"""The file-ingest boundary the validators use (CheckV and viralVerify call
search_hmm_file, BUSCO and EukCC search_hmm_file_models; src/hmmer/search.rs:238-271):
a .hmm library, plain and gzip-compressed (src/hmmer/parse.rs:42-54), of more
than 256 profiles, so the 256-profile batches of search.rs:256-269 are crossed,
searched through the Python mirror of the reference API and loaded whole by
sx_profiles_load_file -- against the oracle's parse and search of the same
bytes."""
import gzip

import numpy as np
import pytest

import sxhmm
from oracle import oracle as O
from sxhmm import synth
from _workloads import oracle_scorer

pytestmark = pytest.mark.gpu

NPROF = 300


@pytest.fixture(scope="module")
def library(tmp_path_factory):
    rng = np.random.default_rng(29)
    profs = [synth.sample_profile(rng, int(rng.integers(20, 80)), f"lib{i:03d}") for i in range(NPROF)]
    synth.calibrate(profs, oracle_scorer, np.random.default_rng(31), nseq=100)
    text = "".join(synth.profile_text(p) for p in profs)
    d = tmp_path_factory.mktemp("hmmlib")
    plain = d / "lib.hmm"
    plain.write_text(text)
    gz = d / "lib.hmm.gz"
    with gzip.open(gz, "wb") as fh:
        fh.write(text.encode())
    seqs = []
    for i in range(40):
        seqs.append((f"bg{i}", synth.residues_to_str(synth.background_seq(rng, int(rng.integers(60, 400))))))
    # homologs of profiles on both sides of the 256-profile batch boundary
    for k in (3, 120, 255, 256, 257, 299):
        dom = synth.emit_homolog(rng, profs[k])
        seqs.append((f"hom{k}", synth.residues_to_str(synth.plant(rng, len(dom) + 80, [dom]))))
    return text, plain, gz, seqs


def _oracle(path, seqs, cfg):
    o = O.Oracle(path=str(path))
    hits, doms = o.search(O.TargetBatch([O.encode(s) for _, s in seqs]), cfg)
    rows = []
    for h in hits:
        ds = [(np.float32(d.score), np.float32(d.bias), d.c_evalue, d.i_evalue, d.hmm_from, d.hmm_to, d.ali_from,
               d.ali_to, d.env_from, d.env_to, bool(d.reported)) for d in doms[h.dom_offset:h.dom_offset + h.ndom]]
        rows.append((o.names[h.profile_index], h.target_index, np.float32(h.score), np.float32(h.bias), h.evalue,
                     np.float32(h.nexpected), ds))
    return o, rows


def _mirror(hits):
    return [(h.profile, h.target_index, np.float32(h.score), np.float32(h.bias), h.evalue, np.float32(h.nexpected),
             [(np.float32(d.score), np.float32(d.bias), d.c_evalue, d.i_evalue, d.hmm_from, d.hmm_to, d.ali_from,
               d.ali_to, d.env_from, d.env_to, bool(d.reported)) for d in h.domains]) for h in hits]


@pytest.mark.parametrize("which", ["plain", "gzip"])
def test_search_hmm_file_models(library, which):
    text, plain, gz, seqs = library
    path = plain if which == "plain" else gz
    eng = sxhmm.Engine()
    try:
        targets = sxhmm.Targets(seqs)
        for cut, ocut in ((sxhmm.Cutoff.evalue(10.0, 10.0), "E"), (sxhmm.Cutoff.gathering(), "GA")):
            cfg = sxhmm.SearchConfig(cut)
            hits, models = sxhmm.search_hmm_file_models(path, targets, cfg, eng)
            o, want = _oracle(path, seqs, O.make_cfg(cutoff=ocut, seq=10.0 if ocut == "E" else 0.0,
                                                      dom=10.0 if ocut == "E" else 0.0))
            assert [(m.name, m.m) for m in models] == list(zip(o.names, o.m))
            assert len(models) == NPROF
            assert _mirror(hits) == want
            if ocut == "E":
                found = {(h[0], seqs[h[1]][0]) for h in want}
                for k in (3, 120, 255, 256, 257, 299):
                    assert (f"lib{k:03d}", f"hom{k}") in found, k
            h2, n = sxhmm.search_hmm_file(path, targets, cfg, eng)
            assert n == NPROF and _mirror(h2) == want
    finally:
        eng.close()


def test_profiles_load_file_plain_and_gzip(library):
    """sx_profiles_load_file reads plain and gzip files alike: the same
    profiles as the text itself and the same search results."""
    text, plain, gz, seqs = library
    eng = sxhmm.Engine()
    try:
        pt = eng.load_text(text)
        ts = eng.targets([s for _, s in seqs])
        cfg = sxhmm.SearchConfig().to_c()
        base = eng.search(pt, ts, cfg)
        for path in (plain, gz):
            pf = eng.load_file(str(path))
            assert len(pf.info) == NPROF
            for a, b in zip(pf.info, pt.info):
                assert a["name"] == b["name"] and a["m"] == b["m"]
            got = eng.search(pf, ts, cfg)
            assert [(h.profile_index, h.target_index, h.score, h.evalue) for h in got[0]] == \
                [(h.profile_index, h.target_index, h.score, h.evalue) for h in base[0]]
            assert len(got[1]) == len(base[1])
        with pytest.raises(sxhmm.HmmError):
            eng.load_file(str(plain) + ".missing")
    finally:
        eng.close()
