"""The N > 1 path of bench.py on CPU: world_size 2 over gloo (127.0.0.1).

The solver path does not shard (replicas only), so what N > 1 adds is the barrier
and the max over ranks of every timing, and the reference arm's rule that rank 0
alone runs and prints while the other ranks exit 0."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r measured (1 + r, 10 - r, 5): the job reports the slowest of each
        vals = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 5.0], dist, "cpu")
        out[rank] = vals
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == [2.0, 10.0, 5.0]


def test_reference_arm_under_torchrun_world2():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--mesh", "16,16,64", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["unit"] == "s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
    # one complete solve to tolerance, not an extrapolated sample
    assert d["cpu_baseline"]["sample"].startswith("measured to tolerance")
    assert d["true_resid"] <= 1e-8 and d["error"] == 0
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_iterations.json")))
    assert d["iterations"] == golden["16,16,64/1"]
