"""Shared inputs for the tests: the reference fixtures, edge-case targets and
small seeded synthetic workloads calibrated with the oracle."""
import functools
import os

import numpy as np

from oracle import oracle as O
from sxhmm import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_text():
    return open(os.path.join(GOLDEN, "hmmer34_pair.hmm")).read()


def tiny_text():
    return open(os.path.join(GOLDEN, "tiny.hmm")).read()


def fixture_targets():
    return O.read_fasta(os.path.join(GOLDEN, "hmmer34_targets.faa"))


oracle_scorer = O.calibration_scorer()


@functools.lru_cache(maxsize=None)
def small_config(idx, scale):
    """A shrunk benchmark config, calibrated with the oracle."""
    return synth.make_config(idx, scale=scale, scorer=oracle_scorer)


def edge_targets():
    """Targets that exercise the edges the reference handles: a single
    residue, degenerate codes, stop/gap characters, lower case, U/O, runs of
    '*', one long sequence."""
    rng = np.random.default_rng(5)
    long = "".join(synth.AA[x] for x in synth.background_seq(rng, 2500))
    return [
        ("one", "M"),
        ("two", "MK"),
        ("degen", "BJZXBJZXMKABJZX"),
        ("stops", "MKA*MKA-MKA.MKA"),
        ("allstop", "****"),
        ("lower_uo", "gggmkaggguuooxxmka"),
        ("motif", "GGGGMKAGGGG"),
        ("two_copies", "GGGGGMKAGGGGGGGGGGGGGGGGGGGGMKAGGGGG"),
        ("long", long),
    ]


def small_profiles_text(seed=3, ms=(1, 2, 5, 33, 64, 65, 129, 300)):
    """Uncalibrated synthetic profiles of awkward lengths (lane/chunk edges)."""
    rng = np.random.default_rng(seed)
    return "".join(synth.profile_text(synth.sample_profile(rng, m, f"edge{m}")) for m in ms)


def long_workload():
    """Profiles longer than the warp-chunked kernels' 2048 columns beside a
    short one (calibrated with the oracle), against background targets,
    planted homologs of both and an empty target."""
    rng = np.random.default_rng(11)
    profs = [synth.sample_profile(rng, 2100, "long2100"), synth.sample_profile(rng, 150, "short150")]
    synth.calibrate(profs, oracle_scorer, np.random.default_rng(7))
    dec = lambda x: "".join(synth.AA[c] for c in x)
    seqs = [(f"bg{i}", dec(synth.background_seq(rng, 300 + 250 * i))) for i in range(5)]
    for i in range(3):
        d = synth.emit_homolog(rng, profs[0])
        seqs.append((f"hom{i}", dec(synth.plant(rng, len(d) + 150, [d]))))
    d = synth.emit_homolog(rng, profs[1])
    seqs.append(("hom_short", dec(synth.plant(rng, 400, [d]))))
    seqs.append(("empty", ""))
    return "".join(synth.profile_text(p) for p in profs), seqs
