"""bench.py --gpus N starts one process per GPU itself when no torchrun
environment is present (world-size-2 gloo ranks on the CPU: the launch and
the exchange, not the GPU work)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_gpus_2_starts_two_ranks():
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--launch-selftest"], capture_output=True, text=True, env=env, timeout=180)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout      # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["world"] == 2 and d["sum"] == 3.0 and d["max_rank"] == 1.0 and d["gpus_arg"] == 2
