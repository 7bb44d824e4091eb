"""Copy the reference's own parity fixtures into tests/golden/.

The reference pins its HMMER engine with test data that lives next to the
Rust sources (src/hmmer/testdata/ of raw-lab/sentinel-x):

* hmmer34_pair.hmm      two calibrated HMMER 3.4 profiles (FAM14 M=378, FAM18 M=218)
* hmmer34_targets.faa   ten target proteins
* hmmer34_expected.tsv  twenty `hmmsearch --max --domtblout` rows from HMMER 3.4
* tiny.hmm              the three-node model of the dp/pipeline/search unit tests

The GPU box has no copy of the reference, so the fixtures are committed here.
They are data, byte-identical to the reference's files; run this script (in a
container that has the reference mounted) to refresh them.  It also records
the known answers asserted by the reference's unit tests (file:line cited) in
unit_expectations.json.
"""
import hashlib
import json
import os
import shutil
import sys

# The reference checkout to copy from, e.g. SX_REFERENCE=/path/to/sentinel-x
REF = os.environ.get("SX_REFERENCE", "")
SRC = os.path.join(REF, "src", "hmmer", "testdata")
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ["hmmer34_pair.hmm", "hmmer34_targets.faa", "hmmer34_expected.tsv", "tiny.hmm"]

# Known answers of the reference's unit tests (inputs and asserted outputs).
UNIT = {
    "alphabet": {  # src/hmmer/alphabet.rs:104-116
        "canonical": ["ACDEFGHIKLMNPQRSTVWY", list(range(20))],
        "uo": ["uo", [1, 8]],
        "degenerate": ["BJZX*", [20, 21, 22, 23, 24]],
        "whitespace": ["m k\n", [10, 8]],
        "bg_sum_tol": 1e-4,
    },
    "parse": {  # src/hmmer/parse.rs:332-370
        "name": "tiny", "acc": "PF99999.1", "m": 3, "ga": [20.0, 18.5], "nc": [10.0, 9.0], "tc": None,
        "mat_1_10": "exp(-0.1)", "t_3_1": 0.0,
        "cutoff_pairs": [["25.00 25.00;", [25.0, 25.0]], ["  792.1 640.3 ;", [792.1, 640.3]], ["30.0 30.0", [30.0, 30.0]]],
    },
    "model": {  # src/hmmer/model.rs:364-393
        "flat_transitions": [0.9, 0.05, 0.05, 0.5, 0.5, 0.5, 0.5],
        "null_l": 300, "null_tol": 1e-3,
    },
    "dp": {  # src/hmmer/dp.rs:916-955
        "fwd_bwd_seq": "GGMKAGGGMKAGG", "fwd_bwd_tol": 1e-3, "matrix_fwd_tol": 1e-4, "matrix_bwd_tol": 1e-3,
        "trace_seq": "GGMKAGGGGGGMKAGG", "trace_domains": [[3, 5, 1, 3], [12, 14, None, None]],
        "vit_le_fwd_slack": 1e-4,
    },
    "pipeline": {  # src/hmmer/pipeline.rs:599-616
        "two_copies_seq": "GGGGGMKAGGGGGGGGGGGGGGGGGGGGMKAGGGGG", "ndom": 2, "first_ali": [6, 8],
    },
    "search": {  # src/hmmer/search.rs:282-305, 316-355
        "bits_targets": [["hit", "GGGGMKAGGGG"], ["miss", "WWWWWWWWWWW"]],
        "parity_tol_bits": 0.1, "parity_rows": 20,
    },
}


def main():
    if not REF:
        sys.exit("set SX_REFERENCE to the reference checkout (the directory holding src/hmmer/testdata)")
    if not os.path.isdir(SRC):
        sys.exit(f"reference testdata not found at {SRC}")
    manifest = {}
    for f in FILES:
        shutil.copyfile(os.path.join(SRC, f), os.path.join(HERE, f))
        manifest[f] = hashlib.sha256(open(os.path.join(HERE, f), "rb").read()).hexdigest()
    with open(os.path.join(HERE, "unit_expectations.json"), "w") as fh:
        json.dump({"source": "src/hmmer/testdata + unit tests of raw-lab/sentinel-x", "sha256": manifest,
                   "unit": UNIT}, fh, indent=1)
    print("wrote", ", ".join(FILES), "and unit_expectations.json")


if __name__ == "__main__":
    main()
