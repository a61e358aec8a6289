"""bench.py's output contract, checked on the CPU through its reference arm (the reference's own CPU path).

One process prints exactly one JSON line with the contract's keys; under the two-process launcher only rank 0
prints and every rank exits 0. The GPU arm's line has the same keys plus the measurement objects; it is produced by
the GPU runs.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def _json_lines(out: str):
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


def _check_line(d, n_gpus):
    if "unavailable" in d:  # the reference could not be built here: a one-line reason is the contract
        assert d["impl"] == "reference" and d["unavailable"]
        return
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["n_gpus"] == n_gpus and d["steps"] == 1 and d["warmup"] == 1
    assert d["value"] > 0 and d["unit"] == "Mparticles/s" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_reference_arm_prints_one_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--cpu-log2n", "12"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1, r.stdout
    _check_line(lines[0], 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_two_ranks_only_rank0_prints():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-log2n", "12"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    if r.returncode != 0 and "torch.distributed" in r.stderr and "rendezvous" in r.stderr.lower():
        pytest.skip("no local rendezvous in this environment")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1, r.stdout
    _check_line(lines[0], 2)
