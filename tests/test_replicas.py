"""Multi-GPU runs of the implicit step are independent replicas: a barrier
around the timed region and the maximum of the ranks' times, nothing on the
data path (dare_b200.replicas, used by bench.py under torchrun).  Two gloo
ranks on CPU processes check that plumbing without a GPU."""
import json
import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from dare_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    slowest = r.max(float(10 * rank + 3))   # rank 1 is the slowest: 13 ms
    steps = 5
    value = r.world * steps / (slowest * 1e-3)  # all ranks' steps over the slowest rank's time
    r.close()
    with open(os.path.join(out, f"r{rank}.json"), "w") as fh:
        json.dump({"rank": r.rank, "world": r.world, "max": slowest, "value": value, "device": r.device}, fh)


def test_two_gloo_replicas(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    res = [json.load(open(tmp_path / f"r{i}.json")) for i in range(2)]
    assert [x["rank"] for x in res] == [0, 1]
    assert all(x["world"] == 2 and x["max"] == 13.0 and x["device"] == "cpu" for x in res)
    assert all(abs(x["value"] - 2 * 5 / 13e-3) < 1e-9 for x in res)


def test_one_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from dare_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.world == 1 and r.dist is None
    assert r.max(4.5) == 4.5
    r.barrier()
    r.close()
