"""sxhmm: B200 hmmsearch engine (Python front end over the C ABI in include/sxhmm.h).

Mirrors the search API of the reference engine (src/hmmer/mod.rs:30,
src/hmmer/search.rs): `Targets`, `SearchConfig`, `PipelineConfig`, `Cutoff`,
`search_profiles`, `search_hmm_file`, `search_hmm_file_models`, `Hit`,
`DomainHit`, `ModelInfo`, with the same field names, argument meaning and
error behaviour (a missing GA/NC/TC cutoff raises with the reference's text).
The compute runs in libsxhmm.so on an sm_100a GPU; there is no CPU fallback:
importing works anywhere, but creating an engine without the library or a
B200 raises.
"""
from ._capi import (SX_CUT_BITS, SX_CUT_EVALUE, SX_CUT_GA, SX_CUT_NC, SX_CUT_TC, Engine, HmmError, LibraryMissing,
                    Profiles, TargetSet, library_path, load_library)
from .search import (Cutoff, DomainHit, Hit, ModelInfo, PipelineConfig, SearchConfig, Targets, default_engine,
                     search_hmm_file, search_hmm_file_models, search_profiles, search_text)

__all__ = [
    "Engine", "Profiles", "TargetSet", "HmmError", "LibraryMissing", "library_path", "load_library",
    "Cutoff", "DomainHit", "Hit", "ModelInfo", "PipelineConfig", "SearchConfig", "Targets", "default_engine",
    "search_hmm_file", "search_hmm_file_models", "search_profiles", "search_text",
    "SX_CUT_EVALUE", "SX_CUT_BITS", "SX_CUT_GA", "SX_CUT_NC", "SX_CUT_TC",
]
