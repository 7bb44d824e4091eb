"""The seeded synthetic workload generator (numpy only)."""
import numpy as np

from oracle import oracle as O
from sxhmm import synth


def test_deterministic_and_parseable():
    a = synth.make_config(0, scale=0.02)
    b = synth.make_config(0, scale=0.02)
    assert a.hmm_text() == b.hmm_text()
    assert all(np.array_equal(x, y) for x, y in zip(a.targets, b.targets))
    o = O.Oracle(text=a.hmm_text())
    assert o.n == 1 and o.m == [100]


def test_shapes_follow_configs():
    w1 = synth.make_config(1, scale=0.01)
    ms, ls = w1.ms, w1.lens
    assert ms.min() >= 20 and ms.max() <= 1000 and ls.min() >= 30 and ls.max() <= 3000
    w3 = synth.make_config(3, scale=1 / 16)
    assert len(w3.pairs) == len(w3.targets) and all(p.m == 300 for p in w3.profiles)


def test_blosum_background_permutation():
    assert abs(synth.BLOSUM_BG.sum() - 1.0) < 1e-9
    # A is first in both orders, W is 18th in HMMER order and 18th in BLOSUM's too
    assert synth.BLOSUM_BG[0] == synth._BLOSUM_BG[0]
    assert synth.BLOSUM_BG[synth.AA.index("R")] == synth._BLOSUM_BG[1]


def test_calibration_with_oracle_scorer():
    from _workloads import small_config
    w = small_config(0, 0.05)
    p = w.profiles[0]
    mmu, vmu, tau, lam = p.stats
    assert abs(lam - np.log(2)) < 1e-12
    assert -20 < mmu < 5 and -20 < vmu < 5 and -20 < tau < 10
    cut, st = O.Oracle(text=w.hmm_text()).header(0)
    assert not np.isnan(st).any()
