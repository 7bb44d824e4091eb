"""Kernel-shape autotuner for the Viterbi filter.

For each range of profile lengths it calibrates synthetic profiles of that
range on the device and runs single-block searches of them against a fixed
set of background targets of the Pfam-scale length distribution, once per
compiled lane-group shape that holds the range's longest profile (G lanes x C
columns, transitions in registers or not), and keeps the shape with the
shortest Viterbi stage (CUDA events, cells / time).  Timing the stage inside
the search matters: its input is the MSV survivor list in the cascade's own
order, which an isolated timing of the kernel on profile-major pairs does not
reproduce.  The result is a table the engine applies to profile sets loaded
afterwards (Engine.set_shape_table), or C source for the built-in default:

    python -m sxhmm.tune --out vit_table.json --emit-inc csrc/tuned_shapes.inc
"""
import argparse
import json
import math

import numpy as np

from . import synth
from ._capi import Engine
from .search import SearchConfig

# upper ends of the profile-length ranges; each range gets one shape
BUCKETS = (32, 64, 96, 128, 160, 192, 256, 320, 384, 512, 640, 768, 1024, 1536, 2048)
MAX_M = 2048


def _targets(engine, rng, n):
    lens = synth.lognormal_lengths(rng, n, 300, synth.SIGMA_L, 30, 3000)
    seqs = [synth.background_seq(rng, int(x)) for x in lens]
    lens = np.array([len(x) for x in seqs], np.int64)
    offs = np.zeros(n, np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    return engine.targets_digital(np.concatenate(seqs).astype(np.uint8), offs, lens), lens


def tune_viterbi(engine, buckets=BUCKETS, nprofiles=48, ntargets=40000, reps=2, seed=5, log=None):
    """Returns (table, report): table[m] = fastest shape index for M = m
    (-1 where no bucket applies), report = per bucket the Viterbi-stage GCUPS
    of every candidate.  `engine` should run single-block searches
    (pipeline_blocks=1) so that the stage is timed alone."""
    rng = np.random.default_rng(seed)
    ts, lens = _targets(engine, rng, ntargets)
    shapes = engine.shapes("viterbi")
    table = np.full(MAX_M + 1, -1, np.int32)
    cfg = SearchConfig().to_c()
    report = []
    lo = 0
    for hi in buckets:
        ms = rng.integers(lo + 1, hi + 1, size=nprofiles)
        profs = [synth.sample_profile(rng, int(m), f"tune{hi}_{i}") for i, m in enumerate(ms)]
        synth.calibrate(profs, synth.engine_scorer(engine), np.random.default_rng(7))
        text = "".join(synth.profile_text(p) for p in profs)
        cands = [i for i, (g, c, _) in enumerate(shapes) if g * c >= hi]
        rates = {}
        for i in cands:
            t = np.full(MAX_M + 1, -1, np.int32)
            t[lo + 1:hi + 1] = i
            engine.set_shape_table("viterbi", t)
            ps = engine.load_text(text, source="tune")
            best, cells = math.inf, 0.0
            for _ in range(reps):
                engine.search(ps, ts, cfg)
                st = engine.stats()
                if st["ms"][2] > 0:
                    best = min(best, st["ms"][2])
                    cells = st["cells"][2]
            ps.close()
            rates[i] = cells / (best / 1e3) / 1e9 if best < math.inf else 0.0
        engine.set_shape_table("viterbi", None)
        win = max(rates, key=rates.get)
        table[lo + 1:hi + 1] = win
        mid = (lo + 1 + hi) // 2
        report.append({"m_range": [lo + 1, hi],
                       "gcups": {f"{shapes[i][0]}x{shapes[i][1]}{'r' if shapes[i][2] else ''}": round(r, 1)
                                 for i, r in rates.items()},
                       "best": list(shapes[win]), "builtin": list(shapes[engine.shape_for("viterbi", mid)])})
        if log:
            log(report[-1])
        lo = hi
    ts.close()
    return table, report


def emit_inc(table, shapes):
    """C source for the built-in table: ranges of M with their (G, C, RT)."""
    rows = []
    m = 1
    while m <= MAX_M:
        s = int(table[m])
        e = m
        while e + 1 <= MAX_M and int(table[e + 1]) == s:
            e += 1
        if s >= 0:
            g, c, rt = shapes[s]
            rows.append(f"    {{{m}, {e}, {g}, {c}, {rt}}},")
        m = e + 1
    rows.append("    {0, -1, 0, 0, 0},")
    return ("// Viterbi lane-group shape per range of profile lengths, measured on B200 by\n"
            "// sentinel-x_b200/sxhmm/tune.py (python -m sxhmm.tune --emit-inc ...).\n"
            "// Rows: first M, last M, G, C, transitions in registers; a row of zeros\n"
            "// applies to no profile.  Ranges without a row keep the cost model's choice.\n"
            "constexpr int kTunedVit[][5] = {\n" + "\n".join(rows) + "\n};\n")


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", help="JSON: the table and the measurements")
    ap.add_argument("--emit-inc", help="C source for the built-in table")
    ap.add_argument("--targets", type=int, default=40000, help="background targets per search")
    a = ap.parse_args()
    eng = Engine(device=a.device, pipeline_blocks=1)
    table, report = tune_viterbi(eng, ntargets=a.targets, log=lambda r: print(json.dumps(r), flush=True))
    shapes = eng.shapes("viterbi")
    if a.out:
        with open(a.out, "w") as f:
            json.dump({"table": table.tolist(), "shapes": shapes, "report": report}, f)
    if a.emit_inc:
        with open(a.emit_inc, "w") as f:
            f.write(emit_inc(table, shapes))
    eng.close()


if __name__ == "__main__":
    main()
