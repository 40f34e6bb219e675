"""The multi-GPU path on CPU: two gloo ranks run bench.py's rank logic
(independent replica sets per rank, the timing barrier, max / sum over
ranks).  The path shards by replicas and has no data exchange, so this is
all the communication there is."""
import json
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, REPO)
    import bench
    rk = bench.Ranks(backend="gloo", timeout_s=60)
    specs = bench.ensemble_specs(32, bench.ENSEMBLE["seed"] + 1000 * rk.rank)
    reqs = bench.served_trace(0.2, bench.SERVED["seed"] + 1000 * rk.rank)
    local_units = float(sum(n for n, _, _, _ in specs))
    local_time = 1.0 + rk.rank  # rank 1 is the slower one
    rk.barrier()
    out = {
        "rank": rk.rank,
        "specs": specs,
        "reqs": [(r.natom, r.seed) for r in reqs],
        "units": rk.sum(local_units),
        "time": rk.max(local_time),
        "local_units": local_units,
    }
    rk.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(out, f)


def test_two_gloo_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    # independent replica sets and traces: the seeds differ per rank
    assert r[0]["specs"] != r[1]["specs"]
    assert {s[3] for s in r[0]["specs"]}.isdisjoint({s[3] for s in r[1]["specs"]})
    assert r[0]["reqs"] != r[1]["reqs"]
    # whole-job value = all ranks' units / the slowest rank's time
    total = r[0]["local_units"] + r[1]["local_units"]
    for k in range(2):
        assert r[k]["units"] == total
        assert r[k]["time"] == 2.0
