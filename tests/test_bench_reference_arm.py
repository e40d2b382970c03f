"""bench.py's reference arm on the CPU: one JSON line with the contract's keys
(impl, metric, value, cpu_baseline, zero-byte e2e), and under
torch.distributed.run with two ranks only rank 0 prints it while the other
rank exits 0 without work.  When the reference build is absent the arm
prints its "unavailable" line instead, which is accepted too."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--cells", "16", "--ref-sample", "8"]


def _json_lines(out: str):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check_line(line):
    assert line["impl"] == "reference"
    if "unavailable" in line:
        return
    assert line["value"] > 0 and line["unit"] == "cell-updates/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_single_process():
    r = subprocess.run([sys.executable, *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0])


def test_reference_arm_two_ranks_rank0_prints():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), *ARGS, "--gpus", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0])
    if "unavailable" not in lines[0]:
        assert lines[0]["n_gpus"] == 2
