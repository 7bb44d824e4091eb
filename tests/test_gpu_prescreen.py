"""The two conservative screens of the device cascade, on the GPU.

* Packed MSV pre-screen (int16x2, two profiles per lane; csrc/prescreen.cuh):
  its bound equals the CPU model of tests/_prescreen_model.py bit for bit, is
  never below the reference's f32 MSV score (src/hmmer/dp.rs:92-145; the
  oracle-pinned score of sx_score_pairs), and searches give the same hits
  with the pre-screen on and off.
* Packed Viterbi pre-screen (int16x2, two targets of one profile per lane;
  csrc/prescreen.cuh vit16_kernel): its bound equals the CPU model bit for
  bit, is never below the reference's f32 Viterbi score (src/hmmer/dp.rs:152-189),
  and searches give the same hits with the pre-screens on and off.
* F3 pre-screen (forward_kernel SCAN order): its Forward score differs from
  the exact (reference-order) Forward score by at most the rounding bound the
  cascade adds to its threshold, (L+1)(2M + 6 VC + 64) 2^-24 nats taken
  twice, on adversarial pairs (M near 2048, L up to 3000, many rescaled rows).
"""
import numpy as np
import pytest

import sxhmm
from oracle import oracle as O
from sxhmm import synth
from _prescreen_model import msv_bound as model_bound
from _prescreen_model import vit_bound as vit_model, vit16_width
from _workloads import edge_targets, fixture_targets, fixture_text, small_config, small_profiles_text, tiny_text

pytestmark = pytest.mark.gpu

LN2 = float(np.float32(0.693147182464599609375))


def _width(engine, m):
    shapes = engine.shapes("msv")
    g, c = shapes[engine.shape_for("msv", m)][:2]
    return g * c


def test_msv_prescreen_bound_model_and_guarantee():
    w = small_config(1, 0.01)
    text = w.hmm_text() + fixture_text() + tiny_text() + small_profiles_text()
    seqs = [synth.residues_to_str(s) for s in w.targets[:120]] + [s for _, s in edge_targets()] + \
        [s for _, s in fixture_targets()]
    o = O.Oracle(text=text)
    e = sxhmm.Engine()
    try:
        ps = e.load_text(text)
        ts = e.targets(seqs)
        pp, pt = np.meshgrid(np.arange(o.n), np.arange(len(seqs)), indexing="ij")
        pp, pt = pp.ravel().astype(np.int32), pt.ravel().astype(np.int32)
        got = e.score_prescreens(ps, ts, pp, pt)["msv_bound"]
        exact = e.score_pairs(ps, ts, pp, pt, stages=("msv",))["msv"]
        dsq = [O.encode(s) for s in seqs]
        arrays = [o.arrays(i) for i in range(o.n)]
        # the guarantee on every pair the pre-screen handles
        handled = ~np.isnan(got)
        assert handled.sum() > 0.9 * len(pp)
        assert np.all(got[handled] >= exact[handled]), np.nonzero(got[handled] < exact[handled])
        # bit-exact with the model on a sample (every profile, every edge target)
        rng = np.random.default_rng(3)
        pick = np.unique(np.concatenate([rng.choice(len(pp), 600, replace=False),
                                         np.nonzero(pt >= 120)[0]]))
        for q in pick:
            i, j = int(pp[q]), int(pt[q])
            a = arrays[i]
            want = model_bound(a["msc"], o.m[i], a["msv_tbm"], _width(e, o.m[i]), dsq[j])
            assert (np.isnan(want) and np.isnan(got[q])) or want == got[q], (i, j, o.m[i], len(dsq[j]), want, got[q])
        # the margin the bound leaves on background pairs stays small
        fin = handled & np.isfinite(got) & np.isfinite(exact)
        slack = got[fin].astype(np.float64) - exact[fin]
        assert np.median(slack) < 0.05, np.median(slack)
    finally:
        e.close()


def test_vit_prescreen_bound_model_and_guarantee():
    """Profiles at every pre-screen width's edges (M 20..513), the config-1
    profiles and the fixture, against background, edge and fixture targets
    and planted homologs strong enough to reach the int16 cap."""
    rng = np.random.default_rng(17)
    w = small_config(1, 0.01)
    extra = [synth.sample_profile(rng, m, f"v{m}") for m in (20, 32, 33, 64, 65, 128, 200, 256, 300, 511, 512, 513)]
    text = w.hmm_text() + "".join(synth.profile_text(p) for p in extra) + fixture_text() + tiny_text()
    seqs = [synth.residues_to_str(s) for s in w.targets[:50]] + [s for _, s in edge_targets()] + \
        [s for _, s in fixture_targets()]
    for p in (extra[1], extra[6], extra[10]):
        dom = synth.emit_homolog(rng, p)
        seqs.append(synth.residues_to_str(synth.plant(rng, len(dom) + 60, [dom])))
    o = O.Oracle(text=text)
    e = sxhmm.Engine()
    try:
        ps = e.load_text(text)
        ts = e.targets(seqs)
        pp, pt = np.meshgrid(np.arange(o.n), np.arange(len(seqs)), indexing="ij")
        pp, pt = pp.ravel().astype(np.int32), pt.ravel().astype(np.int32)
        got = e.score_prescreens(ps, ts, pp, pt)["vit_bound"]
        exact = e.score_pairs(ps, ts, pp, pt, stages=("viterbi",))["viterbi"]
        dsq = [O.encode(s) for s in seqs]
        arrays = [o.arrays(i) for i in range(o.n)]
        handled = ~np.isnan(got)
        wide = np.array([vit16_width(o.m[i]) is None for i in pp])
        empty = np.array([len(dsq[j]) == 0 for j in pt])
        assert not handled[wide | empty].any()
        assert handled.sum() > 0.8 * len(pp)
        # the guarantee on every pair the pre-screen handles
        assert np.all(got[handled] >= exact[handled]), np.nonzero(got[handled] < exact[handled])
        assert np.isinf(got[handled]).any(), "no pair reached the cap"
        # bit-exact with the model on a sample: every profile x every edge,
        # fixture and homolog target, plus random pairs
        rng2 = np.random.default_rng(5)
        pick = np.unique(np.concatenate([rng2.choice(len(pp), 300, replace=False), np.nonzero(pt >= 50)[0]]))
        for q in pick:
            i, j = int(pp[q]), int(pt[q])
            a = arrays[i]
            want = vit_model(a["msc"], a["t"], o.m[i], dsq[j])
            assert (np.isnan(want) and np.isnan(got[q])) or want == got[q], (i, j, o.m[i], len(dsq[j]), want, got[q])
        # the margin on background pairs stays small
        fin = handled & np.isfinite(got) & np.isfinite(exact)
        slack = got[fin].astype(np.float64) - exact[fin]
        print(f"vit bound slack: median {np.median(slack):.3f} nats, 99% {np.quantile(slack, 0.99):.3f}")
        assert np.median(slack) < 1.0, np.median(slack)
    finally:
        e.close()


@pytest.mark.parametrize("cfg,scale", [(0, 1.0), (1, 0.01), (4, 0.002)])
def test_search_prescreen_on_off_identical(cfg, scale):
    w = small_config(cfg, scale)
    text = w.hmm_text()
    lens = np.array([len(s) for s in w.targets], np.int64)
    offs = np.zeros(len(lens), np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    seq = np.concatenate(w.targets).astype(np.uint8)
    out = []
    for pre in (True, False):
        e = sxhmm.Engine(prescreen=pre)
        try:
            ps = e.load_text(text)
            ts = e.targets_digital(seq, offs, lens)
            hits, doms = e.search(ps, ts, sxhmm.SearchConfig().to_c())
            st = e.stats()
            if pre:
                assert st["prescreen"]["pairs_in"] == len(w.profiles) * len(lens)
                assert 0 < st["prescreen"]["pairs_out"] < st["prescreen"]["pairs_in"]
                # the exact kernel saw exactly the pre-screen's survivors and kept what F1 keeps
                assert st["pairs_out"][0] <= st["prescreen"]["pairs_out"]
                # the Viterbi pre-screen bounded bias survivors and passed a subset
                vp = st["vprescreen"]
                assert 0 < vp["pairs_in"] <= st["pairs_out"][1]
                assert vp["pairs_out"] <= vp["pairs_in"]
                assert st["pairs_out"][2] <= vp["pairs_out"] + (st["pairs_out"][1] - vp["pairs_in"])
            else:
                assert st["prescreen"]["pairs_in"] == 0
                assert st["vprescreen"]["pairs_in"] == 0
            out.append(([(h.profile_index, h.target_index, h.score, h.bias, h.evalue, h.ndomains) for h in hits],
                        [(d.score, d.env_from, d.env_to, d.hmm_from, d.hmm_to) for d in doms], st["pairs_out"][0]))
        finally:
            e.close()
    assert out[0] == out[1]


def test_forward_prescreen_rounding_bound():
    """Adversarial pairs for the F3 pre-screen's rounding bound: the widest
    warp-chunked profiles (M 1,950-2,040, 64 columns per lane) and M = 600
    against long targets (L up to 3,000) carrying several planted homologs,
    whose Forward values grow past the 1e4 rescale threshold on many rows."""
    rng = np.random.default_rng(41)
    profs = [synth.sample_profile(rng, m, f"wide{m}") for m in (2040, 1950, 600)]
    text = "".join(synth.profile_text(p) for p in profs)
    seqs = []
    for p in profs:
        for ndom in (1, 3, 5):
            doms = [synth.emit_homolog(rng, p) for _ in range(ndom)]
            total = min(3000, sum(len(d) for d in doms) + 200)
            seqs.append(synth.residues_to_str(synth.plant(rng, total, doms)))
    for L in (300, 1500, 3000):
        seqs.append(synth.residues_to_str(synth.background_seq(rng, L)))
    e = sxhmm.Engine()
    try:
        ps = e.load_text(text)
        ts = e.targets(seqs)
        pp, pt = np.meshgrid(np.arange(len(profs)), np.arange(len(seqs)), indexing="ij")
        pp, pt = pp.ravel().astype(np.int32), pt.ravel().astype(np.int32)
        scan = e.score_prescreens(ps, ts, pp, pt)["fwd_scan"].astype(np.float64)
        exact = e.score_pairs(ps, ts, pp, pt, stages=("forward",))["forward"].astype(np.float64)
        worst = 0.0
        for q in range(len(pp)):
            m, L = profs[pp[q]].m, len(seqs[pt[q]])
            vc = next(v for v in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64) if 32 * v >= m)
            bound_bits = 2.0 * (L + 1) * (2 * m + 6 * vc + 64) * 2.0 ** -24 / LN2
            diff_bits = abs(scan[q] - exact[q]) / LN2
            # 1e-3 bits: the device's log against glibc's (the cascade's slack)
            assert diff_bits <= bound_bits + 1e-3, (m, L, diff_bits, bound_bits)
            worst = max(worst, diff_bits / (bound_bits + 1e-3))
        # homologs drove the Forward values through the rescale threshold
        assert np.nanmax(exact) > 200.0
        print(f"worst |scan - exact| / allowed = {worst:.3g}")
    finally:
        e.close()
