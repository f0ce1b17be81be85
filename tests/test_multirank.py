"""The N > 1 path of bench.py on CPU: two gloo ranks through the same rank
coordination the GPU run uses (process group from the torchrun environment,
barrier, max over ranks), the replica seeds, and the reference arm's
rank-0-only rule.  The GPU run itself is replicas only: no collective touches
the data path, so these host steps are the whole multi-rank logic.
"""

import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench
    w, r, local, dist = bench.init_ranks("gloo", timeout_s=60)
    assert (w, r, local) == (world, rank, rank) and dist is not None
    bench.barrier(dist)
    m = bench.max_over_ranks(1.5 + rank, dist, "cpu")
    bench.barrier(dist)
    Path(out_dir, f"rank{rank}.txt").write_text(repr(m))
    dist.destroy_process_group()


def test_two_gloo_ranks_max_and_barrier(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    vals = [float(Path(tmp_path, f"rank{r}.txt").read_text()) for r in range(world)]
    assert vals == [2.5, 2.5]


def test_single_rank_needs_no_process_group(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    w, r, local, dist = bench.init_ranks("gloo")
    assert (w, r, local, dist) == (1, 0, 0, None)
    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25


@pytest.mark.parametrize("workload", ["akm3", "slopes", "gi", "kss", "ols", "prep", "savefe",
                                      "batch"])
def test_reference_arm_runs_on_rank0_only(monkeypatch, workload):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--workload", workload,
                                      "--steps", "1", "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.main() == 0
    assert buf.getvalue() == ""


def test_replica_panels_differ_by_rank_seed():
    sys.path.insert(0, str(ROOT))
    import bench
    import numpy as np
    a = bench.make_panel(20_000, seed=0)
    b = bench.make_panel(20_000, seed=1)
    assert not np.array_equal(a.y[:100], b.y[:100])
