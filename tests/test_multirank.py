"""The N>1 path of bench.py on CPU: two gloo ranks, each with its own shot.

A multi-GPU job runs one independent shot per rank (there is no data-path collective); the only
exchange is the max-over-ranks of the timed durations, and the whole-job throughput counts every
rank's nodes.  Here each rank advances a different golden shot with the oracle, the ranks agree on
the slowest time through `max_over_ranks`, and each rank's fields equal those of the same shot run
alone -- a rank's result does not depend on the other rank.
"""
import importlib.util
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
SHOTS = ["sponge_force", "cpml_external_moment_layers"]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _load_bench():
    spec = importlib.util.spec_from_file_location("_bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank: int, world: int, port: int, out_dir: str):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_oracle
    from helpers import load_2d

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench = _load_bench()
    case, res, mesh = load_2d(SHOTS[rank])
    steps = 20
    st, _, _, _ = load_oracle().Oracle().run2d(mesh, steps)
    local_ms = 10.0 + 5.0 * rank  # each rank's own (pretend) duration
    slowest = bench.max_over_ranks(local_ms, dist, "cpu")
    points = (int(res["nx"]) - 6) * (int(res["nz"]) - 6)
    np.savez(Path(out_dir) / f"rank{rank}.npz", state=st, slowest=slowest, points=points,
             throughput=bench.job_throughput(points, steps, slowest, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_each_run_their_own_shot(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    world, port = 2, _free_port()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_oracle
    from helpers import load_2d

    orc = load_oracle().Oracle()
    for rank in range(world):
        r = np.load(tmp_path / f"rank{rank}.npz")
        assert float(r["slowest"]) == 15.0  # both ranks see the slowest rank's time
        assert float(r["throughput"]) == pytest.approx(world * int(r["points"]) * 20 / (15.0e-3) / 1e6)
        _, _, mesh = load_2d(SHOTS[rank])
        alone, _, _, _ = orc.run2d(mesh, 20)
        np.testing.assert_array_equal(r["state"], alone)
