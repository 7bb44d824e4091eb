"""CPU checks of the pre-screens' CPU models (tests/_prescreen_model.py)
against the oracle: the bound each model computes -- which the GPU tests pin
the kernels to bit for bit -- is never below the reference's f32 score
(MSV src/hmmer/dp.rs:92-145, Viterbi dp.rs:152-189), on background pairs,
planted homologs, the awkward widths of the kernels' shapes and the edge
targets.  A pair the reference passes through a filter therefore always
passes the pre-screen in front of it."""
import numpy as np

from oracle import oracle as O
from sxhmm import synth
from _prescreen_model import msv_bound, vit_bound, vit16_width
from _workloads import edge_targets


def _setup(seed, ms):
    rng = np.random.default_rng(seed)
    profs = [synth.sample_profile(rng, m, f"p{m}") for m in ms]
    o = O.Oracle(text="".join(synth.profile_text(p) for p in profs))
    seqs = [O.encode(synth.residues_to_str(synth.background_seq(rng, int(L)))) for L in (1, 7, 40, 150, 400)]
    seqs += [O.encode(s) for _, s in edge_targets() if s]
    for p in profs[:3]:
        dom = synth.emit_homolog(rng, p)
        seqs.append(O.encode(synth.residues_to_str(synth.plant(rng, len(dom) + 40, [dom]))))
    return o, seqs


def test_vit_model_bounds_oracle():
    o, seqs = _setup(23, (12, 33, 64, 129, 257, 512))
    worst = 0.0
    for i in range(o.n):
        a = o.arrays(i)
        for d in seqs:
            b = vit_bound(a["msc"], a["t"], o.m[i], d)
            ex = np.float32(o.viterbi(i, d))
            assert vit16_width(o.m[i]) is not None and not np.isnan(b)
            assert b >= ex, (o.m[i], len(d), b, ex)
            if np.isfinite(b) and np.isfinite(ex):
                worst = max(worst, float(b) - float(ex))
    # the bound stays close: rounding up every score by at most 2^-9 nat
    assert worst < 2.0, worst


def test_vit_model_width_limit():
    o, seqs = _setup(29, (513,))
    a = o.arrays(0)
    assert np.isnan(vit_bound(a["msc"], a["t"], 513, seqs[2]))
    assert np.isnan(vit_bound(a["msc"], a["t"], 513, np.zeros(0, np.uint8)))


def test_msv_model_bounds_oracle():
    o, seqs = _setup(31, (12, 33, 150, 400))
    for i in range(o.n):
        a = o.arrays(i)
        for d in seqs:
            b = msv_bound(a["msc"], o.m[i], a["msv_tbm"], 512, d)
            ex = np.float32(o.msv(i, d))
            assert b >= ex, (o.m[i], len(d), b, ex)


def test_vit_model_bounds_oracle_randomised():
    """Random profiles across the pre-screen's widths (M 1-512, the edges of
    every shape included) against random targets that carry degenerate
    residues and '*', lengths 1-400, and planted homologs: the bound is never
    below the oracle's Viterbi score."""
    rng = np.random.default_rng(101)
    ms = [1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512]
    ms += [int(x) for x in rng.integers(4, 512, 8)]
    profs = [synth.sample_profile(rng, m, f"r{i}") for i, m in enumerate(ms)]
    o = O.Oracle(text="".join(synth.profile_text(p) for p in profs))
    alphabet = np.array(list("ACDEFGHIKLMNPQRSTVWYXBZU*"))
    checked = 0
    for i in range(o.n):
        a = o.arrays(i)
        seqs = []
        for _ in range(3):
            L = int(rng.integers(1, 400))
            seqs.append(O.encode("".join(rng.choice(alphabet, L, p=None))))
        dom = synth.emit_homolog(rng, profs[i])
        seqs.append(O.encode(synth.residues_to_str(synth.plant(rng, len(dom) + int(rng.integers(0, 80)), [dom]))))
        for d in seqs:
            b = vit_bound(a["msc"], a["t"], o.m[i], d)
            ex = np.float32(o.viterbi(i, d))
            assert not np.isnan(b)
            assert b >= ex, (o.m[i], len(d), b, ex)
            checked += 1
    assert checked == 4 * len(ms)


def test_msv_model_bounds_oracle_randomised():
    """The MSV pre-screen's bound model against the oracle's f32 MSV on random
    profiles (M 1-2048), random targets with degenerate residues and '*', and
    planted homologs, at the narrowest width a lane-group shape gives and at a
    padded one."""
    rng = np.random.default_rng(202)
    ms = [1, 2, 7, 8, 9, 100, 300, 1000, 2048]
    profs = [synth.sample_profile(rng, m, f"q{i}") for i, m in enumerate(ms)]
    o = O.Oracle(text="".join(synth.profile_text(p) for p in profs))
    alphabet = np.array(list("ACDEFGHIKLMNPQRSTVWYXBZU*"))
    for i in range(o.n):
        a = o.arrays(i)
        m = o.m[i]
        seqs = [O.encode("".join(rng.choice(alphabet, int(rng.integers(1, 300))))) for _ in range(3)]
        dom = synth.emit_homolog(rng, profs[i])
        seqs.append(O.encode(synth.residues_to_str(synth.plant(rng, len(dom) + 40, [dom]))))
        for width in (((m + 7) // 8) * 8, ((m + 63) // 64) * 64 + 64):
            for d in seqs:
                b = msv_bound(a["msc"], m, a["msv_tbm"], width, d)
                ex = np.float32(o.msv(i, d))
                assert b >= ex, (m, width, len(d), b, ex)
