"""bench.py's multi-GPU path on CPU: two gloo ranks, each with its own profile
block against the same targets (weak scaling, no data-path collective); the
job's time is the slowest rank's and its work the sum of the ranks' cells."""
import multiprocessing as mp
import socket

import pytest

import _multirank


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_multirank.worker, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        d = q.get(timeout=300)
        res[d["rank"]] = d
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = res[0], res[1]
    assert a["seq"] == b["seq"], "every rank searches the same targets"
    assert a["text"] != b["text"], "each rank has its own profile block"
    for d in (a, b):
        assert d["ms_max"] == 150.0 and d["e2e_max"] == 300.0
        assert d["cells_total"] == pytest.approx(a["cells"] + b["cells"])
        assert d["value"] == pytest.approx((a["cells"] + b["cells"]) / 0.150 / 1e9)
