"""bench.py --impl reference (the oracle on the host cores) keeps the bench
line contract: one JSON line from rank 0 with the metric, value, e2e and
cpu_baseline keys, at N=1 and under torchrun with two gloo ranks (where rank 1
does no work and exits 0)."""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT, _ensure_oracle

BENCH = os.path.join(ROOT, "bench.py")
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--ref-step-seconds", "0.3"]


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check(line, n_gpus):
    assert line["impl"] == "reference"
    assert line["metric"] == line["unit"] == "Mpaths/s"
    assert line["n_gpus"] == n_gpus and line["steps"] == 1 and line["warmup"] == 1
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "Mpaths/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "1000 flat 10x10 heliostats" in line["config"]["workload"]


def test_reference_arm_one_process():
    _ensure_oracle()
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, BENCH] + ARGS, capture_output=True, text=True,
                       timeout=600, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _lines(p.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_two_ranks():
    _ensure_oracle()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), BENCH, "--gpus", "2"] + ARGS
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _lines(p.stdout)
    assert len(lines) == 1
    _check(lines[0], 2)
