"""The reference's search API (src/hmmer/search.rs) over the B200 engine.

Names and semantics follow src/hmmer/search.rs:24-271: `Cutoff` variants
(Evalue/Bits/Gathering/Noise/Trusted), `SearchConfig{cutoff, pipeline, z}`,
`PipelineConfig{filters, null2, f1, f2, f3}` with HMMER's defaults, `Targets`
of digitised sequences, `Hit`/`DomainHit` records in profile order then target
order, and `search_hmm_file(_models)` streaming a .hmm(.gz) library in batches
of 256 profiles (search.rs:252-271).
"""
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

from . import _capi

_ENGINE = None


def default_engine():
    global _ENGINE
    if _ENGINE is None:
        _ENGINE = _capi.Engine()
    return _ENGINE


@dataclass(frozen=True)
class Cutoff:
    """hmmsearch -E/--domE, -T/--domT, --cut_ga, --cut_nc, --cut_tc (search.rs:26-38)."""
    kind: str = "evalue"
    seq: float = 10.0
    dom: float = 10.0

    @staticmethod
    def evalue(seq=10.0, dom=10.0):
        return Cutoff("evalue", seq, dom)

    @staticmethod
    def bits(seq, dom):
        return Cutoff("bits", seq, dom)

    @staticmethod
    def gathering():
        return Cutoff("gathering", 0.0, 0.0)

    @staticmethod
    def noise():
        return Cutoff("noise", 0.0, 0.0)

    @staticmethod
    def trusted():
        return Cutoff("trusted", 0.0, 0.0)

    def code(self):
        return {"evalue": _capi.SX_CUT_EVALUE, "bits": _capi.SX_CUT_BITS, "gathering": _capi.SX_CUT_GA,
                "noise": _capi.SX_CUT_NC, "trusted": _capi.SX_CUT_TC}[self.kind]


@dataclass
class PipelineConfig:
    """Pipeline switches with HMMER 3.4 defaults (pipeline.rs:27-42)."""
    filters: bool = True
    null2: bool = True
    f1: float = 0.02
    f2: float = 1e-3
    f3: float = 1e-5


@dataclass
class SearchConfig:
    cutoff: Cutoff = field(default_factory=Cutoff)
    pipeline: PipelineConfig = field(default_factory=PipelineConfig)
    z: Optional[float] = None

    def to_c(self):
        p = self.pipeline
        return _capi.search_cfg(self.cutoff.code(), self.cutoff.seq, self.cutoff.dom, p.filters, p.null2, p.f1, p.f2,
                                p.f3, self.z)


class Targets:
    """Target proteins (search.rs:50-80): ids and raw sequences; digitised and
    uploaded to the device when first searched."""

    def __init__(self, pairs):
        self.ids = [str(a) for a, _ in pairs]
        self.seqs = [b.encode() if isinstance(b, str) else bytes(b) for _, b in pairs]
        self._dev = {}

    @classmethod
    def from_pairs(cls, pairs):
        return cls(pairs)

    def __len__(self):
        return len(self.ids)

    def is_empty(self):
        return not self.ids

    def device(self, engine):
        key = id(engine)
        if key not in self._dev:
            self._dev[key] = engine.targets(self.seqs, self.ids)
        return self._dev[key]


@dataclass
class DomainHit:
    score: float
    bias: float
    c_evalue: float
    i_evalue: float
    hmm_from: int
    hmm_to: int
    ali_from: int
    ali_to: int
    env_from: int
    env_to: int
    reported: bool


@dataclass
class Hit:
    profile: str
    acc: Optional[str]
    qlen: int
    target: str
    target_index: int
    tlen: int
    score: float
    bias: float
    evalue: float
    nexpected: float
    domains: List[DomainHit]

    def reported_domains(self):
        return [d for d in self.domains if d.reported]

    def best_domain_score(self):
        return max((d.score for d in self.domains), default=float("-inf"))


@dataclass
class ModelInfo:
    name: str
    acc: Optional[str]
    m: int


def _to_hits(profiles, targets, raw_hits, raw_doms):
    out = []
    for h in raw_hits:
        info = profiles.info[h.profile_index]
        doms = [DomainHit(d.score, d.bias, d.c_evalue, d.i_evalue, d.hmm_from, d.hmm_to, d.ali_from, d.ali_to,
                          d.env_from, d.env_to, bool(d.reported))
                for d in raw_doms[h.domain_offset:h.domain_offset + h.ndomains]]
        out.append(Hit(info["name"], info["acc"], h.qlen, targets.ids[h.target_index], h.target_index, h.tlen,
                       h.score, h.bias, h.evalue, h.nexpected, doms))
    return out


def search_profiles(profiles, targets: Targets, cfg: SearchConfig, engine=None) -> List[Hit]:
    """All profiles x all targets (search.rs:213-234). `profiles` is a
    _capi.Profiles set on the same engine."""
    eng = engine or profiles.engine
    hits, doms = eng.search(profiles, targets.device(eng), cfg.to_c())
    return _to_hits(profiles, targets, hits, doms)


def search_text(text, targets: Targets, cfg: SearchConfig, engine=None) -> List[Hit]:
    eng = engine or default_engine()
    return search_profiles(eng.load_text(text), targets, cfg, eng)


def _split_records(path):
    """Yield the HMMER3 text records of a (gzip) file one at a time."""
    import gzip
    with open(path, "rb") as fh:
        magic = fh.read(2)
    opener = gzip.open if magic == b"\x1f\x8b" else open
    buf = []
    with opener(path, "rt", errors="replace") as fh:
        for line in fh:
            buf.append(line)
            if line.strip() == "//":
                yield "".join(buf)
                buf = []
    if any(l.strip() for l in buf):
        yield "".join(buf)


def search_hmm_file_models(path, targets: Targets, cfg: SearchConfig, engine=None) -> Tuple[List[Hit], List[ModelInfo]]:
    """Stream a .hmm(.gz) file in batches of 256 profiles (search.rs:252-271)."""
    eng = engine or default_engine()
    hits, models, batch = [], [], []

    def flush():
        if not batch:
            return
        ps = eng.load_text("".join(batch), source=str(path))
        models.extend(ModelInfo(i["name"], i["acc"], i["m"]) for i in ps.info)
        hits.extend(search_profiles(ps, targets, cfg, eng))
        ps.close()
        batch.clear()
    for rec in _split_records(path):
        batch.append(rec)
        if len(batch) == 256:
            flush()
    flush()
    return hits, models


def search_hmm_file(path, targets: Targets, cfg: SearchConfig, engine=None) -> Tuple[List[Hit], int]:
    hits, models = search_hmm_file_models(path, targets, cfg, engine)
    return hits, len(models)
