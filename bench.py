"""Benchmark: Plan7 hmmsearch GCUPS on one B200 (Pfam-scale batch).

Workload (the Pfam-scale configuration): 1,000 synthetic Plan7 profiles with
M log-normal (median 150, clipped 20..1,000) against 50,000 synthetic proteins
with L log-normal (median 300, clipped 30..3,000), 2% carrying a planted
homolog; STATS calibrated on the device; default hmmsearch thresholds
(E <= 10, F1 = 0.02, F2 = 1e-3, F3 = 1e-5).  A step is one full search
(every profile x every target through MSV -> bias -> Viterbi -> Forward,
Backward, domain definition and reporting).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value  = sum over pairs of M*L / device time of the step (inputs resident on
         the device, L2 flushed between steps), whole job over all ranks.
e2e    = same metric through the public C ABI with host buffers: digitised
         targets copied host->device, search, hits read back, every step.
         The profile set stays loaded on the device across steps, as a
         library serving a stream of searches keeps it (loading it once per
         profile file is the reference's use too: search_hmm_file parses a
         library once per call, then searches every target batch).
Under torchrun (N > 1) each rank searches its own block of 1,000 profiles
against the same targets (profile-block sharding, no data-path collective).
"""
import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

# The engine drives up to 31 streams (two pipeline slots, high- and
# low-priority sets, and the domain passes' copy stream); give the process 32 hardware work queues before
# anything initialises CUDA, so high-priority stages never queue behind MSV.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sentinel-x_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Plan7 GCUPS (MSV/Vit/Fwd/Bwd), batched vs plain on 1 B200; hits bit-exact"
STAGES = ["msv", "bias", "viterbi", "forward", "rows", "host_domains", "total", "host_tail"]
WORKLOAD = ("pfam_scale: 1000 profiles M~LN(150,0.5)[20,1000] x 50000 targets L~LN(300,0.6)[30,3000], "
            "2% planted homologs, E<=10, F1/F2/F3 = 0.02/1e-3/1e-5")
MSV_OPS_PER_CELL = 3  # 1 FADD + 2 FMAX per cell (src/hmmer/dp.rs:122-124)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sxhmm", choices=["sxhmm", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="shrink profile/target counts (testing only)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain one-pair-per-block kernels")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip timing sx_posterior_grad on the adjoint workload (4,096 pairs, M=300, L>=400)")
    ap.add_argument("--marker-genomes", type=int, default=10,
                    help="genomes of the marker-set configuration searched one by one (100 = all; 0 = skip)")
    ap.add_argument("--no-prescreen", action="store_true",
                    help="run the exact MSV kernel on every pair (no packed pre-screen), for comparison")
    ap.add_argument("--pipeline-blocks", type=int, default=0,
                    help="profile blocks per search (0 = engine default by workload size)")
    return ap.parse_args()


_T0 = time.time()


def progress(msg):
    """Phase marker on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write(f"[bench {time.time() - _T0:7.1f}s] {msg}\n")
    sys.stderr.flush()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_seed(rank):
    """Seed of rank `rank`'s profile block: rank 0 searches the single-GPU
    workload, rank r > 0 a block of the same size drawn with its own seed."""
    return None if rank == 0 else 1001 + 7919 * rank


def reduce_max(vals, dist, device):
    """Per-value maximum over ranks (identity without a process group)."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def reduce_sum(vals, dist, device):
    """Per-value sum over ranks (identity without a process group)."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def whole_job_gcups(total_cells, ms):
    """Aggregate throughput: all ranks' DP cells over the slowest rank's time."""
    return total_cells / (ms / 1e3) / 1e9


def workload(scale, rank, scorer=None):
    from sxhmm import synth
    cache = os.environ.get("SXHMM_BENCH_CACHE", "/tmp/sxhmm_bench_cache")
    os.makedirs(cache, exist_ok=True)
    key = os.path.join(cache, f"cfg1_s{scale}_r{rank}.npz")
    if os.path.exists(key):
        z = np.load(key, allow_pickle=False)
        return str(z["text"]), z["seq"], z["offs"], z["lens"], int(z["ntarg"])
    w = synth.make_config(1, scale=scale, seed=rank_seed(rank), scorer=scorer)
    if rank:
        # every rank searches the same targets with its own profile block
        w0 = synth.make_config(1, scale=scale)
        w.targets = w0.targets
    text = w.hmm_text()
    lens = w.lens
    offs = np.zeros(len(lens), np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    seq = np.concatenate(w.targets).astype(np.uint8)
    np.savez(key, text=np.array(text), seq=seq, offs=offs, lens=lens, ntarg=len(lens))
    return text, seq, offs, lens, len(lens)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def sha1(text):
    import hashlib
    return hashlib.sha1(text.encode()).hexdigest()[:16]


def cpu_baseline(text, seq, offs, lens, seconds, as_line=False):
    """The oracle's threaded driver (a C++ restatement of the reference's
    rayon pair loop) on a bounded, deterministic sample of the workload: 2,000
    strided targets x every profile in profile-major order, stopped after
    `seconds` of wall time (about 11 s of 16-thread work when it runs out)."""
    from oracle import oracle as O
    o = O.Oracle(text=text)
    nt = len(lens)
    cfg = O.make_cfg()
    # sample: a strided subset of targets, all profiles (so M covers the distribution)
    ms = np.array(o.m, dtype=np.float64)
    stride = max(1, nt // 2000)
    pick = np.arange(0, nt, stride)[:2000]
    sub = O.TargetBatch([seq[offs[i]:offs[i] + lens[i]] for i in pick])
    threads = os.cpu_count() or 1
    r = o.time_pairs(sub, cfg, nthreads=threads, time_limit=seconds)
    gcups = r["cells"] / r["seconds"] / 1e9 if r["seconds"] > 0 else None
    return {"value": gcups, "unit": "GCUPS", "cores": threads, "kind": "port",
            "sample": f"{r['pairs']} pairs ({r['cells']:.3e} cells) of {len(pick)} strided targets x "
                      f"{o.n} profiles (profile-major), oracle score_target pipeline, {r['seconds']:.1f} s",
            "pairs": r["pairs"], "seconds": r["seconds"]}


def sample_targets(seq, offs, lens, n=2000):
    """The deterministic target sample of the CPU legs: n targets at a fixed
    stride through the workload, packed back to back."""
    nt = len(lens)
    stride = max(1, nt // n)
    pick = np.arange(0, nt, stride)[:n]
    sub = [seq[offs[i]:offs[i] + lens[i]] for i in pick]
    slens = np.array([len(x) for x in sub], np.int64)
    soffs = np.zeros(len(sub), np.int64)
    soffs[1:] = np.cumsum(slens)[:-1]
    return pick, np.concatenate(sub).astype(np.uint8), soffs, slens


def _hit_rows(hits, doms, oracle_side):
    """Hits and their domains as comparable tuples: every field of the
    reference's Hit / DomainHit that both sides report (f32 scores, f64
    E-values, coordinates, reported flags)."""
    rows = []
    for h in hits:
        off, nd = (h.dom_offset, h.ndom) if oracle_side else (h.domain_offset, h.ndomains)
        ds = [(np.float32(d.score).item(), np.float32(d.bias).item(), float(d.c_evalue), float(d.i_evalue),
               d.hmm_from, d.hmm_to, d.ali_from, d.ali_to, d.env_from, d.env_to, int(bool(d.reported)))
              for d in doms[off:off + nd]]
        rows.append((h.profile_index, h.target_index, np.float32(h.score).item(), np.float32(h.bias).item(),
                     float(h.evalue), np.float32(h.nexpected).item(), ds))
    return rows


def oracle_leg(eng, ps, text, seq, offs, lens):
    """CPU baseline and full-size parity in one pass: the oracle's threaded
    search (the reference's rayon pair loop restated: score_target on every
    pair, then report) over the 2,000-target sample x every profile, timed on
    all host threads; the engine searches the same targets with the same
    profile set, and the two hit lists are compared field by field with ==."""
    from oracle import oracle as O
    import sxhmm
    o = O.Oracle(text=text)
    pick, sseq, soffs, slens = sample_targets(seq, offs, lens)
    sub = O.TargetBatch.from_packed(sseq, soffs, slens)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ohits, odoms = o.search(sub, O.make_cfg(), nthreads=threads)
    secs = time.perf_counter() - t0
    ms = np.array(o.m, dtype=np.float64)
    cells = float(ms.sum()) * float(slens.sum())
    ts = eng.targets_digital(sseq, soffs, slens)
    ghits, gdoms = eng.search(ps, ts, sxhmm.SearchConfig().to_c())
    ts.close()
    a = _hit_rows(ohits, odoms, True)
    b = _hit_rows(ghits, gdoms, False)
    mismatch = None
    if len(a) != len(b):
        mismatch = f"{len(a)} oracle hits vs {len(b)} engine hits"
    else:
        for x, y in zip(a, b):
            if x != y:
                mismatch = f"oracle {x[:6]} vs engine {y[:6]}"
                break
    parity = {"pairs": int(o.n * len(slens)), "targets": int(len(slens)), "profiles": int(o.n),
              "hits": len(a), "domains": int(sum(len(x[6]) for x in a)), "identical": mismatch is None,
              "compared": "profile, target, score, bias, E-value, nexpected; per domain score, bias, c/i-Evalue, "
                          "hmm/ali/env coordinates, reported (==)",
              "z": "number of targets in the sample (2,000), on both sides"}
    if mismatch:
        parity["first_mismatch"] = mismatch
    base = {"value": cells / secs / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
            "sample": f"{o.n * len(slens)} pairs ({cells:.3e} cells) of {len(slens)} strided targets x {o.n} "
                      f"profiles, full oracle search (score_target pipeline + report), {secs:.1f} s"}
    return base, parity


def flush_l2(torch, buf):
    buf.add_(1.0)  # 256 MiB write > 126 MB L2


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    text, seq, offs, lens, nt = workload(args.scale, 0, scorer=O.calibration_scorer())
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(text, seq, offs, lens, max(2.0, args.cpu_seconds / max(1, args.steps)))
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([x["value"] for x in vals])
    line = {"metric": METRIC, "value": v, "unit": "GCUPS", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": vals[-1]["sample"], "hmm_sha1": sha1(text)},
            "cpu_baseline": {k: vals[-1][k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["cpu_baseline"]["value"] = v
    print(json.dumps(line), flush=True)


def adjoint_run(sxhmm, eng, torch):
    """sx_posterior_grad (lnZ and the expected counts of every emission and
    transition, sqrt(L) checkpointed) on the adjoint workload: 16 profiles of
    M = 300, 256 targets each (L >= 400, 0-3 planted domains)."""
    from sxhmm import synth
    cache = os.environ.get("SXHMM_BENCH_CACHE", "/tmp/sxhmm_bench_cache")
    os.makedirs(cache, exist_ok=True)
    key = os.path.join(cache, "cfg3.npz")
    if os.path.exists(key):
        z = np.load(key, allow_pickle=False)
        text, seq, offs, lens, pp, pt = str(z["text"]), z["seq"], z["offs"], z["lens"], z["pp"], z["pt"]
    else:
        w = synth.make_config(3)
        text = w.hmm_text()
        lens = np.array([len(t) for t in w.targets], np.int64)
        offs = np.zeros(len(lens), np.int64)
        offs[1:] = np.cumsum(lens)[:-1]
        seq = np.concatenate(w.targets).astype(np.uint8)
        pp = np.array([a for a, _ in w.pairs], np.int32)
        pt = np.array([b for _, b in w.pairs], np.int32)
        np.savez(key, text=np.array(text), seq=seq, offs=offs, lens=lens, pp=pp, pt=pt)
    ps = eng.load_text(text, source="adjoint")
    ts = eng.targets_digital(seq, offs, lens)
    cells = float(sum(300 * int(lens[t]) for t in pt))
    grads = eng.posterior_grad(ps, ts, pp, pt, 300)  # warm-up; its arrays are reused, as a training loop would
    ms = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.posterior_grad(ps, ts, pp, pt, 300, out=grads)
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
    # homolog-heavy search on the same data (hmmsearch --max: every one of the
    # 16 x 4,096 pairs reaches domain definition): envelope rescoring and the
    # stochastic traces of multi-domain regions on the device, envelopes on
    # the device with traces on the host, the engine's own choice, and all on
    # the host (the adjoint profiles carry no STATS, so a bit-score cutoff
    # reports the hits)
    cfg_max = sxhmm.SearchConfig(sxhmm.Cutoff.bits(0.0, 0.0), sxhmm.PipelineConfig(filters=False)).to_c()
    dom = {}
    for where, envelopes, traces in (("device", "device", "device"), ("device_host_traces", "device", "host"),
                                     ("auto", "auto", "auto"), ("host", "host", "auto")):
        e2 = sxhmm.Engine(device=torch.cuda.current_device(), envelopes=envelopes, traces=traces)
        ps2 = e2.load_text(text, source="adjoint")
        ts2 = e2.targets_digital(seq, offs, lens)
        e2.search(ps2, ts2, cfg_max)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hits, doms = e2.search(ps2, ts2, cfg_max)
        torch.cuda.synchronize()
        st = e2.stats()
        dom[where] = {"ms": round((time.perf_counter() - t0) * 1e3, 1), "hits": len(hits), "domains": len(doms),
                      "envelopes_on_device": st["pairs_out"][5], "regions_traced_on_device": st["pairs_out"][6],
                      "regions_redone_on_host": st["pairs_in"][6] - st["pairs_out"][6],
                      "host_busy_ms": round(st["ms"][5], 1), "host_tail_ms": round(st["ms"][7], 1)}
        ps2.close()
        ts2.close()
        e2.close()
    ps.close()
    ts.close()
    t = statistics.median(ms)
    return {"pairs": int(len(pp)), "cells": cells, "ms": round(t, 1), "gcups": round(cells / (t / 1e3) / 1e9, 1),
            "domain_search": dom,
            "what": "lnZ + gradients w.r.t. all match/insert emission and transition scores per pair "
                    "(Forward with sqrt(L) checkpoints, Backward with segment recomputation); host arrays "
                    "out (the caller's, reused across calls), copies included"}


def marker_set_run(sxhmm, local, torch, ngenomes, prescreen=True, envelopes="auto", traces="auto", batch_bytes=0):
    """The marker-set configuration as BUSCO and EukCC issue it
    (src/busco/mod.rs:297-304, src/eukcc/mod.rs:77): 250 marker profiles
    (M uniform 200-1,500) against one genome of 4,000 proteins at a time
    (L log-normal, median 280, clipped 30-4,000), each marker planted once in
    90% of genomes and twice in 5%, gathering cutoffs, filters on.  Every
    genome is one search through the C ABI with its proteins copied from host
    memory and its hits read back; the first `ngenomes` genomes of the full
    100-genome draw are searched.  Reports the per-genome wall time beside
    the engine's device stage times and its launch count, whose difference
    bounds the host-side launch and synchronisation cost a CUDA-graph replay
    could remove."""
    from sxhmm import synth
    cache = os.environ.get("SXHMM_BENCH_CACHE", "/tmp/sxhmm_bench_cache")
    os.makedirs(cache, exist_ok=True)
    key = os.path.join(cache, f"cfg2_g{ngenomes}.npz")
    eng = sxhmm.Engine(device=local, prescreen=prescreen, envelopes=envelopes, traces=traces, batch_bytes=batch_bytes)
    t0 = time.time()
    if os.path.exists(key):
        z = np.load(key, allow_pickle=False)
        text, seq, offs, lens, gen = str(z["text"]), z["seq"], z["offs"], z["lens"], z["gen"]
    else:
        w = synth.make_config(2, genomes=ngenomes, scorer=synth.engine_scorer(eng))
        text = w.hmm_text()
        lens = np.array([len(t) for t in w.targets], np.int64)
        offs = np.zeros(len(lens), np.int64)
        offs[1:] = np.cumsum(lens)[:-1]
        seq = np.concatenate(w.targets).astype(np.uint8)
        gen = np.array(w.truth["genomes"], np.int64)
        np.savez(key, text=np.array(text), seq=seq, offs=offs, lens=lens, gen=gen)
    gen_s = time.time() - t0
    ps = eng.load_text(text, source="marker_set")
    ms = np.array([i["m"] for i in ps.info], dtype=np.float64)
    cfg = sxhmm.SearchConfig(sxhmm.Cutoff.gathering()).to_c()
    pinned = torch.from_numpy(seq).pin_memory().numpy()

    def genome(g):
        g0, n = int(gen[g][0]), int(gen[g][1])
        o = offs[g0:g0 + n] - offs[g0]
        a, b = int(offs[g0]), int(offs[g0 + n - 1] + lens[g0 + n - 1])
        return pinned[a:b], o, lens[g0:g0 + n]

    s0, o0, l0 = genome(0)
    ts = eng.targets_digital(s0, o0, l0)
    eng.search(ps, ts, cfg)  # warm-up
    ts.close()
    walls, launches, hits, cells = [], [], 0, 0.0
    stage = np.zeros(8)
    pin, pout = np.zeros(8), np.zeros(8)
    pre_ms = res_ms = vpre_ms = 0.0
    for g in range(len(gen)):
        sg, og, lg = genome(g)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ts = eng.targets_digital(sg, og, lg)
        h, d = eng.search(ps, ts, cfg)
        walls.append((time.perf_counter() - t) * 1e3)
        ts.close()
        st = eng.stats()
        stage += np.array(st["ms"])
        pin += np.array(st["pairs_in"])
        pout += np.array(st["pairs_out"])
        pre_ms += st["prescreen"]["ms"]
        res_ms += st["prescreen"]["rescore_ms"]
        vpre_ms += st["vprescreen"]["ms"]
        launches.append(st["kernel_launches"])
        hits += len(h)
        cells += float(ms.sum()) * float(lg.sum())
    ng = len(gen)
    per = {k: round(v / ng, 2) for k, v in zip(STAGES, stage)}
    wall = statistics.median(walls)
    # device stages on the critical path of one genome's search: the MSV stage,
    # then bias, Viterbi, the Forward pre-screen and the row passes one after
    # the other, then the host's work after the last device stage
    critical = per["msv"] + per["bias"] + per["viterbi"] + per["forward"] + per["rows"] + per["host_tail"]
    eng.close()
    return {"workload": "marker_set: 250 profiles M~U[200,1500] x genomes of 4000 proteins L~LN(280,0.6)[30,4000], "
                        "markers planted once in 90% / twice in 5% of genomes, Cutoff::Gathering, filters on",
            "genomes": ng, "cells": cells, "hits": hits, "generation_s": round(gen_s, 1),
            "gcups": round(cells / (sum(walls) / 1e3) / 1e9, 1),
            "wall_ms_per_genome": {"median": round(wall, 2), "min": round(min(walls), 2), "max": round(max(walls), 2)},
            "stage_ms_per_genome": per,
            "prescreen_ms_per_genome": round(pre_ms / ng, 2), "rescore_ms_per_genome": round(res_ms / ng, 2),
            "viterbi_prescreen_ms_per_genome": round(vpre_ms / ng, 2),
            "launches_per_genome": int(statistics.median(launches)),
            "per_genome": {"final_pairs": round(pin[4] / ng, 1), "envelopes_on_device": round(pout[5] / ng, 1),
                           "regions_to_device": round(pin[6] / ng, 1), "regions_traced_on_device": round(pout[6] / ng, 1)},
            "placement": {"envelopes": envelopes, "traces": traces},
            "host_gap_ms_per_genome": round(max(0.0, wall - critical), 2),
            "host_gap_note": "median wall (target upload + search + hits) minus the device stages on the critical "
                             "path (MSV, bias, Viterbi, Forward pre-screen, row passes) and the host tail (which "
                             "includes the envelopes' device passes): an upper bound on launch, copy and "
                             "synchronisation overhead per search; 0 when those stages already cover the wall time "
                             "(they overlap, so their sum can exceed it)"}


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import sxhmm
    from sxhmm import synth
    eng = sxhmm.Engine(device=local, pipeline_blocks=args.pipeline_blocks, prescreen=not args.no_prescreen)
    t0 = time.time()
    progress("engine created; building the workload")
    text, seq, offs, lens, nt = workload(args.scale, rank, scorer=synth.engine_scorer(eng))
    progress("workload ready")
    gen_s = time.time() - t0
    ps = eng.load_text(text, source="pfam_scale")
    ms = np.array([i["m"] for i in ps.info], dtype=np.float64)
    cells = float(ms.sum()) * float(lens.sum())
    ts = eng.targets_digital(seq, offs, lens)
    cfg = sxhmm.SearchConfig().to_c()
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident steps ----
    progress("device-resident steps")
    for _ in range(args.warmup):
        eng.search(ps, ts, cfg)
    # the interpreter's cyclic garbage collector stays off in the timed loops: a
    # full collection over the workload's Python objects is a pause of this
    # harness (tens of ms), not of the engine
    gc.collect()
    gc.freeze()
    gc.disable()
    sampler = ClockSampler(local)
    sampler.start()
    times, launches, nhits = [], 0, 0
    stage_ms = np.zeros(8)
    stage_pairs = None
    for _ in range(args.steps):
        flush_l2(torch, l2)
        barrier()
        torch.cuda.synchronize()
        ev0.record()
        hits, doms = eng.search(ps, ts, cfg)
        ev1.record()
        torch.cuda.synchronize()
        barrier()
        times.append(ev0.elapsed_time(ev1))
        st = eng.stats()
        stage_ms += np.array(st["ms"])
        launches = st["kernel_launches"]
        stage_pairs = st["pairs_in"][:6]
        nhits = len(hits)
    clocks = sampler.stop()
    # ---- end-to-end steps through the C ABI with host buffers ----
    progress("end-to-end steps")
    e2e_times, e2e_upload, e2e_stage, e2e_parts = [], [], [], []
    h2d = int(seq.nbytes + offs.nbytes + lens.nbytes)
    d2h = 0
    pinned = torch.from_numpy(seq).pin_memory().numpy()
    for step in range(1 + max(1, args.steps)):  # the first pass is an untimed warm-up
        flush_l2(torch, l2)
        barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        ts2 = eng.targets_digital(pinned, offs, lens)
        t_up = time.perf_counter()
        hits2, doms2 = eng.search(ps, ts2, cfg)
        t_se = time.perf_counter()
        torch.cuda.synchronize()
        t_sy = time.perf_counter()
        ts2.close()
        t_cl = time.perf_counter()
        torch.cuda.synchronize()
        if step == 0:
            continue
        e2e_times.append((time.perf_counter() - t) * 1e3)
        e2e_upload.append((t_up - t) * 1e3)
        e2e_parts.append([round((t_se - t_up) * 1e3, 1), round((t_sy - t_se) * 1e3, 1), round((t_cl - t_sy) * 1e3, 1)])
        e2e_stage.append({k: round(v, 1) for k, v in zip(STAGES, eng.stats()["ms"])})
        d2h = len(hits2) * 48 + len(doms2) * 56
    gc.enable()
    progress("single-block searches")
    # ---- MSV kernel alone: a single-block search, where MSV does not share the
    # GPU with later stages of another block, gives the kernel's own event time ----
    reng = sxhmm.Engine(device=local, pipeline_blocks=1, prescreen=not args.no_prescreen)
    rps = reng.load_text(text, source="pfam_scale")
    rts = reng.targets_digital(seq, offs, lens)
    reng.search(rps, rts, cfg)  # warm-up
    msv_ms, msv_cells, single_ms, pre, vpre, vit_ms = [], [], [], [], [], []
    for _ in range(2):
        flush_l2(torch, l2)
        torch.cuda.synchronize()
        ev0.record()
        reng.search(rps, rts, cfg)
        ev1.record()
        torch.cuda.synchronize()
        single_ms.append(ev0.elapsed_time(ev1))
        rst = reng.stats()
        msv_ms.append(rst["ms"][0])
        msv_cells.append(rst["cells"][0])
        pre.append(rst["prescreen"])
        vpre.append(rst["vprescreen"])
        vit_ms.append(rst["ms"][2])
    # stage GCUPS (cells entering a stage / its device time), single-block search
    stage_gcups = {k: round(rst["cells"][i] / (rst["ms"][i] / 1e3) / 1e9, 1) if rst["ms"][i] > 0 else None
                   for k, i in (("msv", 0), ("viterbi", 2), ("forward", 3), ("fwd_bwd_rows", 4))}
    stage_cells = {k: rst["cells"][i] for k, i in (("msv", 0), ("viterbi", 2), ("forward", 3), ("fwd_bwd_rows", 4))}
    rps.close()
    rts.close()
    reng.close()
    # ---- the plain one-pair-per-block kernels on the same inputs ----
    progress("plain kernels" if not args.no_plain else "plain kernels skipped")
    plain = None
    if not args.no_plain:
        peng = sxhmm.Engine(device=local, plain=True, pipeline_blocks=args.pipeline_blocks)
        pps = peng.load_text(text, source="pfam_scale")
        pts = peng.targets_digital(seq, offs, lens)
        phits, _ = peng.search(pps, pts, cfg)  # warm-up
        ptimes = []
        for _ in range(max(1, min(args.steps, 2))):
            flush_l2(torch, l2)
            torch.cuda.synchronize()
            ev0.record()
            phits, _ = peng.search(pps, pts, cfg)
            ev1.record()
            torch.cuda.synchronize()
            ptimes.append(ev0.elapsed_time(ev1))
        pst = peng.stats()
        # end to end as the batched arm's e2e: the targets copied from pinned
        # host memory, the search, the hits read back
        flush_l2(torch, l2)
        torch.cuda.synchronize()
        t = time.perf_counter()
        pts2 = peng.targets_digital(pinned, offs, lens)
        phits2, pdoms2 = peng.search(pps, pts2, cfg)
        torch.cuda.synchronize()
        pe2e_ms = (time.perf_counter() - t) * 1e3
        pts2.close()
        plain = {"value": cells / (max(ptimes) / 1e3) / 1e9, "ms_per_step": max(ptimes), "hits": len(phits),
                 "e2e": {"value": cells / (pe2e_ms / 1e3) / 1e9, "unit": "GCUPS", "ms": round(pe2e_ms, 1),
                         "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": len(phits2) * 48 + len(pdoms2) * 56},
                 "stage_ms": {k: round(v, 3) for k, v in zip(STAGES, pst["ms"])},
                 "what": "one 128-thread CTA per pair, row split across threads, shared-memory exchange + "
                         "__syncthreads per row, block max-reduction, Viterbi D chain by one thread; same "
                         "Forward/Backward/host stages"}
        pps.close()
        pts.close()
        peng.close()
    # K timed steps: per-step CUDA-event times summed (the L2 flush between
    # steps stays outside), divided by K
    ms_step = sum(times) / len(times) if times else float("nan")
    e2e_ms = sum(e2e_times) / len(e2e_times)
    # the job takes as long as its slowest rank; its work is every rank's cells
    ms_step, e2e_ms = reduce_max([ms_step, e2e_ms], dist, "cuda")
    (total_cells,) = reduce_sum([cells], dist, "cuda")
    value = whole_job_gcups(total_cells, ms_step)
    e2e_value = whole_job_gcups(total_cells, e2e_ms)
    # roofline of the dominant kernel (MSV): algorithmic lane-ops per launch / event time
    # The dominant kernel is the packed MSV pre-screen (msv16_kernel), which
    # bounds every pair's MSV score; the exact f32 MSV kernel then rescores the
    # pairs whose bound passes F1.  Its algorithmic work is the reference's MSV
    # work over the cells it covers (3 lane-ops per cell); two profiles share
    # each 32-bit lane, so it can exceed half of the scalar lane peak.
    pre_ms = statistics.median([x["ms"] for x in pre])
    pre_cells = statistics.median([x["cells"] for x in pre])
    if pre_ms > 0:
        msv_t = pre_ms / 1e3
        kernel_cells = pre_cells
        kernel_name = "msv16_kernel (packed int16x2 MSV pre-screen, 2 profiles per lane)"
        smem_bytes = 2.0  # one int16 score per cell
    else:
        msv_t = statistics.median(msv_ms) / 1e3
        kernel_cells = statistics.median(msv_cells)
        kernel_name = "msv_kernel"
        smem_bytes = 4.0
    achieved = MSV_OPS_PER_CELL * kernel_cells / msv_t / 1e12
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    peak = 148 * 128 * sm_mhz * 1e6 / 1e12  # 32-bit lanes x SMs x sampled SM clock
    # the kernel's second ceiling: every DP cell reads its emission score from
    # shared memory, 128 bytes per clock per SM
    smem_achieved = smem_bytes * kernel_cells / msv_t / 1e12
    smem_peak = 148 * 128 * sm_mhz * 1e6 / 1e12
    prescreen = {"pairs_in": pre[-1]["pairs_in"], "pairs_passed": pre[-1]["pairs_out"],
                 "pass_fraction": pre[-1]["pairs_out"] / max(1, pre[-1]["pairs_in"]),
                 "prescreen_ms": round(pre_ms, 3), "rescore_ms": round(statistics.median([x["rescore_ms"] for x in pre]), 3),
                 "msv_stage_ms": round(statistics.median(msv_ms), 3),
                 "gcups": round(pre_cells / (pre_ms / 1e3) / 1e9, 1) if pre_ms > 0 else None}
    # the packed Viterbi pre-screen in front of the exact Viterbi (stage 2)
    vp_ms = statistics.median([x["ms"] for x in vpre])
    vit_prescreen = {"pairs_in": vpre[-1]["pairs_in"], "pairs_passed": vpre[-1]["pairs_out"],
                     "pass_fraction": vpre[-1]["pairs_out"] / max(1, vpre[-1]["pairs_in"]),
                     "prescreen_ms": round(vp_ms, 3), "viterbi_stage_ms": round(statistics.median(vit_ms), 3),
                     "gcups": round(vpre[-1]["cells"] / (vp_ms / 1e3) / 1e9, 1) if vp_ms > 0 else None}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "msv_traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("bytes_per_launch_full")
        except Exception:
            traffic = None
    line = {"metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "profiles_per_rank": int(len(ms)), "targets": int(nt),
                       "cells_per_rank": cells, "parallelism": f"profile-block x{ws}" if ws > 1 else "single GPU",
                       "l2": "flushed between steps (256 MiB write)", "calibration": "on device, 200 x L=100 per profile",
                       "generation_s": round(gen_s, 1), "hits": nhits, "hmm_sha1": sha1(text)},
            "roofline": {"bound": "alu", "kernel": kernel_name, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_note": "148 SMs x 128 32-bit lanes x median sampled SM clock (lane-ops/s); "
                                      "achieved = 3 MSV lane-ops per cell (src/hmmer/dp.rs:122-124) x cells / time",
                         "kernel_ms": round(msv_t * 1e3, 3),
                         "measured_in": "single-block search (pipeline_blocks=1): MSV launches alone on the GPU, "
                                        "CUDA events around them",
                         "single_block_ms_per_step": round(max(single_ms), 3)},
            "roofline_shared": {"bound": "shared memory", "kernel": kernel_name, "achieved": smem_achieved,
                                "peak": smem_peak, "unit": "TB/s", "frac": smem_achieved / smem_peak,
                                "note": f"{smem_bytes:.0f} B of emission score read from shared memory per DP cell; "
                                        "peak 128 B per clock per SM x 148 SMs x median sampled SM clock"},
            "msv_prescreen": prescreen,
            "viterbi_prescreen": vit_prescreen,
            "stage_ms": {k: round(v / max(1, args.steps), 3) for k, v in zip(STAGES, stage_ms)},
            "stage_pairs_in": dict(zip(["msv", "bias", "viterbi", "forward", "rows", "host_domains"], stage_pairs or [])),
            "stage_gcups": stage_gcups, "stage_cells": stage_cells,
            "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps_ms": [round(x, 1) for x in e2e_times],
                    "target_upload_ms": [round(x, 1) for x in e2e_upload],
                    "stage_ms_per_step": e2e_stage, "search_close_ms": e2e_parts},
            "steps_ms": [round(x, 1) for x in times],
            "gpu_launches": int(launches), "clocks": clocks}
    if not args.no_adjoint:
        progress("adjoint workload")
        line["adjoint"] = adjoint_run(sxhmm, eng, torch)
    if args.marker_genomes > 0:
        progress("marker-set workload")
        line["marker_set"] = marker_set_run(sxhmm, local, torch, args.marker_genomes, prescreen=not args.no_prescreen)
    if plain is not None:
        line["plain"] = plain
        line["batched_over_plain"] = plain["ms_per_step"] / ms_step
        line["batched_over_plain_e2e"] = plain["e2e"]["ms"] / e2e_ms
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        progress("oracle leg (CPU baseline + full-size parity)")
        line["cpu_baseline"], line["parity"] = oracle_leg(eng, ps, text, seq, offs, lens)
        progress("oracle leg done")
    if rank == 0:
        print(json.dumps(line), flush=True)
    ps.close()
    ts.close()
    eng.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
