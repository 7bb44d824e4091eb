"""Worker of test_multirank_cpu: one gloo rank of bench.py's multi-GPU path."""
import hashlib
import os
from datetime import timedelta


def worker(rank, ws, port, cache, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank), SXHMM_BENCH_CACHE=cache)
    import numpy as np
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        import bench
        from oracle import oracle as O
        assert bench.dist_env() == (ws, rank, rank)
        text, seq, offs, lens, nt = bench.workload(0.004, rank, scorer=O.calibration_scorer())
        o = O.Oracle(text=text)
        cells = float(np.sum(o.m)) * float(np.sum(lens))
        ms = 100.0 + 50.0 * rank  # this rank's step time: the job's is the slowest rank's
        ms_max, e2e_max = bench.reduce_max([ms, 2 * ms], dist, "cpu")
        (cells_total,) = bench.reduce_sum([cells], dist, "cpu")
        out_q.put(dict(rank=rank, text=hashlib.sha1(text.encode()).hexdigest(),
                       seq=hashlib.sha1(seq.tobytes()).hexdigest(), cells=cells, ms_max=ms_max,
                       e2e_max=e2e_max, cells_total=cells_total,
                       value=bench.whole_job_gcups(cells_total, ms_max)))
    finally:
        dist.destroy_process_group()
