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


def _fleet_rank(rank: int, world: int, port: int, out_dir: str):
    """One rank of a request stream sharded over `world` devices: every rank computes the same
    placement plan from the request list and the budgets alone, and serves its own slot's shots
    (here: builds their models, SWL_MODEL_ONLY, without a GPU).  The ranks exchange nothing on the
    data path; the plan is compared across ranks only to check that it is the same everywhere."""
    import importlib
    import pickle

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_package

    load_package()
    F = importlib.import_module("swl_b200.fleet")
    S = importlib.import_module("swl_b200.session")
    W = importlib.import_module("swl_b200.workloads")
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    reqs = FLEET_REQUESTS(W)
    budget = 3 * max(F.request_bytes(r["params"], r["dim"]) for r in reqs)
    slots = F.plan(reqs, [budget] * world)
    plans = [None] * world
    dist.all_gather_object(plans, slots)
    mine = {}
    for i, (r, s) in enumerate(zip(reqs, slots)):
        if s != rank:
            continue
        sim = (S.Simulation2D if r["dim"] == 2 else S.Simulation3D)(r["params"], device=S.MODEL_ONLY)
        info = sim.info()
        mine[i] = (info["dt"], info["total_steps"], info["nx"], info["nz"])
    with open(Path(out_dir) / f"fleet{rank}.pkl", "wb") as f:
        pickle.dump({"plans": plans, "mine": mine}, f)
    dist.barrier()
    dist.destroy_process_group()


def FLEET_REQUESTS(W):
    return [r for r in W.serving_mix(n=16, scale=0.25, steps_scale=0.01) if r["dim"] == 2][:10]


def test_two_ranks_shard_a_request_stream(tmp_path):
    import importlib
    import pickle

    mp = pytest.importorskip("torch.multiprocessing")
    world, port = 2, _free_port()
    mp.start_processes(_fleet_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_package

    load_package()
    S = importlib.import_module("swl_b200.session")
    W = importlib.import_module("swl_b200.workloads")
    got = [pickle.load(open(tmp_path / f"fleet{r}.pkl", "rb")) for r in range(world)]
    assert got[0]["plans"][0] == got[0]["plans"][1] == got[1]["plans"][0]  # one plan everywhere
    served = {}
    for r in range(world):
        assert not set(served) & set(got[r]["mine"])                        # no request served twice
        served.update(got[r]["mine"])
    reqs = FLEET_REQUESTS(W)
    assert sorted(served) == list(range(len(reqs)))                          # every request served once
    assert all(len(g["mine"]) > 0 for g in got)                              # both ranks have work
    for i, r in enumerate(reqs):                                             # as if run alone
        info = S.Simulation2D(r["params"], device=S.MODEL_ONLY).info()
        assert served[i] == (info["dt"], info["total_steps"], info["nx"], info["nz"])
