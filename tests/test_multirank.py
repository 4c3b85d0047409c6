"""The bench's multi-rank plumbing on CPU (gloo, world size 2): bench.py runs
one independent replica of the case per rank ("replicas only": the path has
no data exchange), brackets the timed region with barriers and reports the
whole job from the slowest rank's time (max over ranks)."""
import os
import sys
import tempfile
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, ws, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "SIMLAB_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_init()
    assert (w, r) == (ws, rank) and dist.get_backend() == "gloo"
    bench.barrier(w)
    # each replica reports its own time; the job's time is the slowest one
    t = bench.max_over_ranks(10.0 + 5.0 * rank, w)
    cells, steps = 1000, 20
    mlups = cells * steps * w / (t * 1e-3) / 1e6
    Path(out_dir, f"r{rank}").write_text(f"{t} {mlups}")
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(2, port, d), nprocs=2, join=True)
        res = [Path(d, f"r{k}").read_text().split() for k in range(2)]
    for t, mlups in res:
        assert float(t) == 15.0
        assert float(mlups) == pytest.approx(1000 * 20 * 2 / 15e-3 / 1e6)
