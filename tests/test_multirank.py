"""The N > 1 path of bench.py on CPU: ranks are gloo processes on this host.

The hot path does not shard (one level per GPU; --gpus N runs N independent
replicas), so the multi-rank logic is the timing aggregation (max over ranks)
and the reference arm's "rank 0 runs, the others exit" rule."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _agg_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = [5.0, 8.0][rank]
    value, t_max = bench.aggregate_mlups(1000, 10, local_ms, world, torch.device("cpu"))
    bench.barrier(world)
    (Path(out_dir) / f"r{rank}.json").write_text(json.dumps([value, t_max]))
    dist.destroy_process_group()


def test_aggregation_takes_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_agg_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        value, t_max = json.loads((tmp_path / f"r{r}.json").read_text())
        assert t_max == 8.0
        assert abs(value - 2 * 1000 * 10 / 8e-3 / 1e6) < 1e-12


def test_reference_arm_runs_on_rank0_only():
    """torchrun with two CPU ranks: exactly one JSON line, printed by rank 0,
    for a small sphere level through the reference CPU path."""
    env = dict(os.environ, ILBM_BENCH_BACKEND="gloo", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1", "--nx", "32", "--ny", "16", "--nz", "16"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0
