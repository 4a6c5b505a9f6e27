"""The N > 1 launch contract on CPU: bench.py under torch.distributed.run with
two ranks over gloo (the reference arm, which needs no GPU).  Rank 0 alone
runs the sample and prints the one JSON line; rank 1 exits 0 without work;
both take part in the final barrier and tear the process group down."""
import json
import os
import pathlib
import socket
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_reference_arm(lib, orc):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--case", "channel", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--ref-seconds", "0.5"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["steps"] == 1
    assert out["value"] > 0 and out["cpu_baseline"]["kind"] == "port"
    assert out["e2e"]["h2d_bytes_per_step"] == 0
