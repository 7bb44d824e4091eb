"""Seeded synthetic Plan7 profiles and target proteins for the hmmsearch path.

The reference publishes no benchmark data for its HMMER engine, and the real
databases its validators search (Pfam, CheckV, BUSCO, EukCC) are not
available, so workloads are synthetic with the shapes the benchmark configs
name:

* match emissions per node ~ Dirichlet(0.5 x BLOSUM62 background), the
  background of src/protsearch/alphabet.rs:86-107 (ARNDCQEGHILKMFPSTWYV order)
  permuted to HMMER's ACDEFGHIKLMNPQRSTVWY order;
* insert emissions = HMMER's background (src/hmmer/alphabet.rs:36-39), which is
  also the residue distribution of background targets;
* transitions per node: (MM, MI, MD) ~ Dir(c(0.9, 0.05, 0.05)),
  (IM, II) ~ Dir(c(0.6, 0.4)), (DM, DD) ~ Dir(c(0.6, 0.4)) with concentration
  c = 20; node 0 has DM = 1, DD = 0 and node M has MD = 0, DM = 1, DD = 0, the
  conventions of HMMER3 files;
* lengths log-normal with sigma_M = 0.5 and sigma_L = 0.6 around the configs'
  medians, clipped to their ranges; numpy PCG64 seed = 1000 + config index;
* homologs: a local path through the core model (entry in the first tenth of
  the nodes, exit in the last tenth, M/I/D moves drawn from the node
  transitions, match residues from the node emissions, insert residues from
  the background) spliced into a background protein;
* STATS LOCAL MSV/VITERBI/FORWARD by simulation: lambda = ln 2; mu for MSV and
  Viterbi by Gumbel maximum likelihood with known lambda over the bit scores of
  200 random L=100 background sequences; tau for Forward by HMMER's p7_Tau
  construction (Gumbel mu of the Forward bit scores, then
  tau = mu - ln(-ln(1 - 0.04))/lambda + ln(0.04)/lambda);
* GA/TC/NC cutoff lines (25/20, 30/25, 20/15 bits) so --cut_* are exercised.

Profiles are written as HMMER3/f text (-ln p with five decimals, '*' for 0),
so the product's parser and the oracle read the same bytes.
"""
import math

import numpy as np

AA = "ACDEFGHIKLMNPQRSTVWY"
# HMMER background, src/hmmer/alphabet.rs:36-39
BG = np.array([0.0787945, 0.0151600, 0.0535222, 0.0668298, 0.0397062, 0.0695071, 0.0229198, 0.0590092, 0.0594422,
               0.0963728, 0.0237718, 0.0414386, 0.0482904, 0.0395639, 0.0540978, 0.0683364, 0.0540687, 0.0673417,
               0.0114135, 0.0304133])
# BLOSUM62 background, src/protsearch/alphabet.rs:86-107, order ARNDCQEGHILKMFPSTWYV
_BLOSUM_ORDER = "ARNDCQEGHILKMFPSTWYV"
_BLOSUM_BG = [0.07421620506799341, 0.05161448614128464, 0.044645808512757915, 0.05362600083855441,
              0.02468745716794485, 0.03425965059141602, 0.0543119256845875, 0.074146941452645, 0.026212984805266227,
              0.06791736761895376, 0.09890786849715096, 0.05815568230307968, 0.02499019757964311,
              0.04741845974228475, 0.038538003320306206, 0.05722902947649442, 0.05089136455028703,
              0.013029956129972148, 0.03228151231375858, 0.07291909820561925]
BLOSUM_BG = np.array([_BLOSUM_BG[_BLOSUM_ORDER.index(a)] for a in AA])
CONC = 20.0
SIGMA_M = 0.5
SIGMA_L = 0.6
LN2 = math.log(2.0)
CUTOFFS = {"GA": (25.0, 20.0), "TC": (30.0, 25.0), "NC": (20.0, 15.0)}


class Profile:
    """A probability-space Plan7 model: mat (M+1,20), ins (M+1,20), t (M+1,7)."""

    def __init__(self, name, mat, ins, t, stats=None, acc=None):
        self.name = name
        self.acc = acc
        self.mat = mat
        self.ins = ins
        self.t = t
        self.stats = stats  # (msv_mu, vit_mu, fwd_tau, lambda) or None
        self.m = mat.shape[0] - 1

    def occupancy(self):
        m, t = self.m, self.t
        occ = np.zeros(m + 1)
        occ[1] = t[0, 1] + t[0, 0]
        for k in range(2, m + 1):
            occ[k] = occ[k - 1] * (t[k - 1, 0] + t[k - 1, 1]) + (1.0 - occ[k - 1]) * t[k - 1, 5]
        return occ

    def compo(self):
        occ = self.occupancy()[1:]
        c = (occ[:, None] * self.mat[1:]).sum(0)
        return c / c.sum()


def sample_profile(rng, m, name, conc=CONC):
    mat = np.zeros((m + 1, 20))
    mat[1:] = rng.dirichlet(0.5 * BLOSUM_BG, size=m)
    # Dirichlet(0.5*bg) occasionally underflows a row to all zeros; floor tiny values
    mat[1:] = np.maximum(mat[1:], 1e-30)
    mat[1:] /= mat[1:].sum(1, keepdims=True)
    ins = np.tile(BG / BG.sum(), (m + 1, 1))
    t = np.zeros((m + 1, 7))
    t[:, 0:3] = rng.dirichlet(conc * np.array([0.9, 0.05, 0.05]), size=m + 1)
    t[:, 3:5] = rng.dirichlet(conc * np.array([0.6, 0.4]), size=m + 1)
    t[:, 5:7] = rng.dirichlet(conc * np.array([0.6, 0.4]), size=m + 1)
    t[0, 5], t[0, 6] = 1.0, 0.0
    mm_mi = t[m, 0] + t[m, 1]
    t[m, 0], t[m, 1], t[m, 2] = t[m, 0] / mm_mi, t[m, 1] / mm_mi, 0.0
    t[m, 5], t[m, 6] = 1.0, 0.0
    return Profile(name, mat, ins, t)


def _fmt_row(v):
    with np.errstate(divide="ignore"):
        nl = -np.log(v)
    return "  ".join("*".rjust(7) if not np.isfinite(x) else f"{x:7.5f}" for x in nl)


def write_hmm_text(name, m, mat_rows, t_rows, stats=None, cutoffs=True, compo=None, acc=None):
    """HMMER3/f text for one profile.  mat_rows: M rows of 20 probabilities
    (nodes 1..M); t_rows: M+1 rows of 7 transition probabilities (nodes 0..M)."""
    mat = np.asarray(mat_rows, dtype=np.float64)
    t = np.asarray(t_rows, dtype=np.float64)
    ins = BG / BG.sum()
    out = ["HMMER3/f [3.4 | synthetic]", f"NAME  {name}"]
    if acc:
        out.append(f"ACC   {acc}")
    out += [f"LENG  {m}", "ALPH  amino"]
    if cutoffs:
        for k, (a, b) in CUTOFFS.items():
            out.append(f"{k}    {a:.2f} {b:.2f};")
    if stats is not None:
        mmu, vmu, ftau, lam = stats
        out.append(f"STATS LOCAL MSV      {mmu:8.4f}  {lam:7.5f}")
        out.append(f"STATS LOCAL VITERBI  {vmu:8.4f}  {lam:7.5f}")
        out.append(f"STATS LOCAL FORWARD  {ftau:8.4f}  {lam:7.5f}")
    out.append("HMM          " + "        ".join(AA))
    out.append("            m->m     m->i     m->d     i->m     i->i     d->m     d->d")
    if compo is None:
        compo = mat.mean(0)
    out.append("  COMPO   " + _fmt_row(np.asarray(compo)))
    out.append("          " + _fmt_row(ins))
    out.append("          " + _fmt_row(t[0]))
    for k in range(1, m + 1):
        out.append(f"  {k:5d}   " + _fmt_row(mat[k - 1]) + f" {k:6d} x - - -")
        out.append("          " + _fmt_row(ins))
        out.append("          " + _fmt_row(t[k]))
    out.append("//")
    return "\n".join(out) + "\n"


def profile_text(p, cutoffs=True):
    return write_hmm_text(p.name, p.m, p.mat[1:], p.t, stats=p.stats, cutoffs=cutoffs, compo=p.compo(), acc=p.acc)


def background_seq(rng, n, freqs=None):
    f = BG / BG.sum() if freqs is None else freqs
    return rng.choice(20, size=n, p=f).astype(np.uint8)


def _cdf(p):
    """The cumulative table numpy's Generator.choice(n, p=p) draws from."""
    c = p.cumsum()
    c /= c[-1]
    return c


def _walk_tables(p):
    """Per-node cumulative tables of emit_homolog's draws (cached on p)."""
    tab = getattr(p, "_walk", None)
    if tab is None:
        m = p.m
        mat = [None] + [_cdf(p.mat[k]) for k in range(1, m + 1)]
        ins = [_cdf(p.ins[k]) for k in range(m + 1)]
        tm = [_cdf(p.t[k][0:3] / p.t[k][0:3].sum()) for k in range(m + 1)]
        ti = [_cdf(p.t[k][3:5] / p.t[k][3:5].sum()) for k in range(m + 1)]
        td = [_cdf(p.t[k][5:7] / p.t[k][5:7].sum()) for k in range(m + 1)]
        tab = p._walk = (mat, ins, tm, ti, td)
    return tab


def emit_homolog(rng, p):
    """Digitised residues of one local path through p (entry in the first tenth
    of the nodes, exit in the last tenth).  Every draw is the one
    rng.choice(n, p=...) makes (one uniform, the first cumulative entry above
    it), from tables computed once per profile."""
    m = p.m
    k = int(rng.integers(1, max(1, m // 10) + 1))
    kend = int(rng.integers(m - m // 10, m + 1)) if m >= 10 else m
    kend = max(kend, k)
    mat, ins, tm, ti, td = _walk_tables(p)
    out = []
    st = 0  # 0 M, 1 I, 2 D
    guard = 0
    while guard < 20 * m + 100:
        guard += 1
        if st == 0:
            out.append(int(mat[k].searchsorted(rng.random(), side="right")))
        elif st == 1:
            out.append(int(ins[k].searchsorted(rng.random(), side="right")))
        if k >= kend:
            break
        if st == 0:
            nxt = int(tm[k].searchsorted(rng.random(), side="right"))
            st, k = (0, k + 1) if nxt == 0 else (1, k) if nxt == 1 else (2, k + 1)
        elif st == 1:
            nxt = int(ti[k].searchsorted(rng.random(), side="right"))
            st, k = (0, k + 1) if nxt == 0 else (1, k)
        else:
            nxt = int(td[k].searchsorted(rng.random(), side="right"))
            st, k = (0, k + 1) if nxt == 0 else (2, k + 1)
    return np.array(out, dtype=np.uint8)


def lognormal_lengths(rng, n, median, sigma, lo, hi):
    v = np.exp(np.log(median) + sigma * rng.standard_normal(n))
    return np.clip(np.rint(v), lo, hi).astype(np.int64)


def plant(rng, total_len, domains, freqs=None):
    """Background protein of ~total_len residues carrying `domains` (list of
    uint8 arrays) at random non-overlapping positions."""
    dl = sum(len(d) for d in domains)
    nbg = max(total_len - dl, len(domains) + 1)
    bg = background_seq(rng, nbg, freqs)
    cuts = np.sort(rng.integers(0, nbg + 1, size=len(domains)))
    parts, prev = [], 0
    for c, d in zip(cuts, domains):
        parts.append(bg[prev:c])
        parts.append(d)
        prev = c
    parts.append(bg[prev:])
    return np.concatenate(parts).astype(np.uint8)


def residues_to_str(dsq):
    return "".join(AA[x] for x in dsq)


# ---------------------------------------------------------------- calibration
def gumbel_mu_known_lambda(x, lam):
    x = np.asarray(x, dtype=np.float64)
    x = x[np.isfinite(x)]
    return -math.log(np.mean(np.exp(-lam * x))) / lam


def calibrate(profiles, scorer, rng, nseq=200, L=100):
    """Fill p.stats for every profile.  scorer(profiles, seqs) must return
    three arrays (len(profiles), len(seqs)) of MSV, Viterbi and Forward scores
    in nats for every (profile, sequence) pair; the null score for length L is
    subtracted here."""
    seqs = [background_seq(rng, L) for _ in range(nseq)]
    msv, vit, fwd = scorer(profiles, seqs)
    p1 = L / (L + 1.0)
    nullsc = L * math.log(p1) + math.log(1.0 - p1)
    lam = LN2
    for i, p in enumerate(profiles):
        mmu = gumbel_mu_known_lambda((np.asarray(msv[i]) - nullsc) / LN2, lam)
        vmu = gumbel_mu_known_lambda((np.asarray(vit[i]) - nullsc) / LN2, lam)
        gmu = gumbel_mu_known_lambda((np.asarray(fwd[i]) - nullsc) / LN2, lam)
        tailp = 0.04
        tau = gmu - math.log(-math.log(1.0 - tailp)) / lam + math.log(tailp) / lam
        p.stats = (mmu, vmu, tau, lam)
    return profiles


# ---------------------------------------------------------------- workloads
class Workload:
    """Profiles (with text), digitised targets and optional explicit pairs."""

    def __init__(self, name, profiles, targets, target_ids, pairs=None, truth=None):
        self.name = name
        self.profiles = profiles
        self.targets = targets
        self.target_ids = target_ids
        self.pairs = pairs
        self.truth = truth or {}

    @property
    def ms(self):
        return np.array([p.m for p in self.profiles], dtype=np.int64)

    @property
    def lens(self):
        return np.array([len(t) for t in self.targets], dtype=np.int64)

    def cells(self):
        if self.pairs is not None:
            ms, ls = self.ms, self.lens
            return float(sum(ms[a] * ls[b] for a, b in self.pairs))
        return float(self.ms.sum()) * float(self.lens.sum())

    def hmm_text(self):
        return "".join(profile_text(p) for p in self.profiles)


def make_config(idx, scale=1.0, scorer=None, seed=None, calib_rng_seed=7, genomes=None):
    """Build benchmark config `idx` (0..4).  scale < 1 shrinks the counts of
    profiles and targets (never their lengths) for quick tests.  For the
    marker-set config (2), `genomes` keeps only the first n genomes of the
    full draw (the same profiles and the same first n genomes)."""
    rng = np.random.default_rng(1000 + idx if seed is None else seed)
    genomes_keep = genomes
    profiles, targets, ids, pairs, truth = [], [], [], None, {}
    if idx == 0:
        profiles = [sample_profile(rng, 100, "synth0_p0")]
        nt = max(2, int(1000 * scale))
        lens = rng.integers(100, 501, size=nt)
        for t in range(nt):
            if rng.random() < 0.05:
                d = emit_homolog(rng, profiles[0])
                targets.append(plant(rng, int(lens[t]), [d]))
                truth.setdefault("homologs", []).append((0, t))
            else:
                targets.append(background_seq(rng, int(lens[t])))
            ids.append(f"t{t}")
    elif idx in (1, 4):
        npf = max(1, int((1000 if idx == 1 else 16000) * scale))
        nt = max(2, int((50000 if idx == 1 else 200000) * scale))
        if idx == 1:
            ms = lognormal_lengths(rng, npf, 150, SIGMA_M, 20, 1000)
            ls = lognormal_lengths(rng, nt, 300, SIGMA_L, 30, 3000)
            hom = 0.02
            freqs = None
        else:
            ms = lognormal_lengths(rng, npf, 180, SIGMA_M, 30, 800)
            ls = lognormal_lengths(rng, nt, 150, SIGMA_L, 40, 1500)
            hom = 0.01
            f = BG * (1.0 + rng.uniform(-0.2, 0.2, size=20))
            freqs = f / f.sum()
        profiles = [sample_profile(rng, int(m), f"synth{idx}_p{i}") for i, m in enumerate(ms)]
        for t in range(nt):
            if rng.random() < hom:
                pi = int(rng.integers(0, npf))
                targets.append(plant(rng, int(ls[t]), [emit_homolog(rng, profiles[pi])], freqs))
                truth.setdefault("homologs", []).append((pi, t))
            else:
                targets.append(background_seq(rng, int(ls[t]), freqs))
            ids.append(f"t{t}")
    elif idx == 2:
        npf = max(1, int(250 * scale))
        ngen = max(1, int(100 * scale))
        nper = max(2, int(4000 * scale))
        ms = rng.integers(200, 1501, size=npf)
        profiles = [sample_profile(rng, int(m), f"marker{i}") for i, m in enumerate(ms)]
        genomes = []
        for g in range(ngen if genomes_keep is None else min(ngen, genomes_keep)):
            ls = lognormal_lengths(rng, nper, 280, SIGMA_L, 30, 4000)
            prots = [background_seq(rng, int(x)) for x in ls]
            for pi in range(npf):
                u = rng.random()
                copies = 1 if u < 0.90 else (2 if u < 0.95 else 0)
                for _ in range(copies):
                    j = int(rng.integers(0, nper))
                    d = emit_homolog(rng, profiles[pi])
                    prots[j] = plant(rng, max(len(prots[j]), len(d) + 20), [d])
                    truth.setdefault("planted", []).append((g, pi, j))
            genomes.append((len(targets), len(prots)))
            for j, s in enumerate(prots):
                targets.append(s)
                ids.append(f"g{g}_{j}")
        truth["genomes"] = genomes
    elif idx == 3:
        npf = max(1, int(16 * scale))
        nper = max(1, int(256 * scale))
        profiles = [sample_profile(rng, 300, f"adj{i}") for i in range(npf)]
        pairs = []
        for pi in range(npf):
            for s in range(nper):
                nd = int(rng.integers(0, 4))
                doms = [emit_homolog(rng, profiles[pi]) for _ in range(nd)]
                dl = sum(len(d) for d in doms)
                seq = plant(rng, max(400, dl + nd + 1), doms) if nd else background_seq(rng, 400)
                targets.append(seq)
                ids.append(f"a{pi}_{s}")
                pairs.append((pi, len(targets) - 1))
    else:
        raise ValueError(idx)
    wl = Workload(f"config{idx}", profiles, targets, ids, pairs, truth)
    if scorer is not None:
        calibrate(profiles, scorer, np.random.default_rng(calib_rng_seed))
    return wl


def engine_scorer(engine):
    """Calibration scorer that runs on the B200 engine: MSV, Viterbi and
    Forward scores of every (profile, sequence) pair via sx_score_pairs."""
    def score(profiles, seqs):
        text = "".join(profile_text(p, cutoffs=False) for p in profiles)
        ps = engine.load_text(text, source="<calibration>")
        lens = np.array([len(s) for s in seqs], dtype=np.int64)
        offs = np.zeros(len(seqs), dtype=np.int64)
        offs[1:] = np.cumsum(lens)[:-1]
        ts = engine.targets_digital(np.concatenate(seqs).astype(np.uint8), offs, lens)
        pp, pt = np.meshgrid(np.arange(len(profiles), dtype=np.int32), np.arange(len(seqs), dtype=np.int32),
                             indexing="ij")
        sc = engine.score_pairs(ps, ts, pp.ravel(), pt.ravel(), stages=("msv", "viterbi", "forward"))
        shape = (len(profiles), len(seqs))
        ps.close()
        ts.close()
        return sc["msv"].reshape(shape), sc["viterbi"].reshape(shape), sc["forward"].reshape(shape)
    return score
