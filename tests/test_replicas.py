"""The multi-GPU path (replicas: independent systems / requests sharded over ranks) on CPU:
two gloo ranks in child processes, the sharding, the max / sum over ranks, a sharded serving
stream (every request served exactly once across ranks), and bench.py's reference arm under
torchrun (rank 0 prints the one JSON line, the other rank exits 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_item_once_and_balances_rows():
    from honei_b200 import replicas
    rng = __import__("numpy").random.default_rng(1)
    sizes = [int(v) for v in rng.integers(17, 1025, 200) ** 2]
    for ws in (1, 2, 3, 8):
        parts = replicas.shard(sizes, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert all(p == sorted(p) for p in parts)
    assert replicas.shard(sizes, 4) == replicas.shard(sizes, 4)


def _rank_main(rank, ws, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from honei_b200 import replicas, serve
    got_ws, got_rank, _ = replicas.init("gloo", timeout_s=60)
    res = {"ws": got_ws, "rank": got_rank, "max": replicas.max_over_ranks(rank + 1.5),
           "sum": replicas.sum_over_ranks(rank + 1)}
    trace = serve.poisson_trace(9, rate=0.0, side_range=(17, 300), seed=3)
    mine = replicas.my_share(trace.requests, [r.M * r.M for r in trace.requests], got_rank, got_ws)
    with serve.Server(mode="mixed", budget_bytes=1 << 30, small_max_side=64, pinned=False) as srv:
        rep = serve.replay(srv, serve.Trace(mine, 0.0, 3, trace.side_range, trace.coef_range), realtime=False)
    tags = [c.tag for c in rep["records"]]
    res["completed_total"] = replicas.sum_over_ranks(len(tags))
    gathered = [None] * got_ws
    dist.all_gather_object(gathered, tags)
    res["all_tags"] = sorted(t for part in gathered for t in part)
    replicas.barrier()
    replicas.finish()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_shard_a_serving_stream(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, d in enumerate(res):
        assert d["ws"] == 2 and d["rank"] == r
        assert d["max"] == 2.5 and d["sum"] == 3.0
        assert d["completed_total"] == 9.0
        assert d["all_tags"] == list(range(9))


def test_bench_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] in ("reference", "port")
