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
    assert "g++ -O3" in d["cpu_baseline"]["build"]  # the compiler flags and CPU model of the timed build
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


def test_summary_is_last_and_fits_the_kept_tail():
    """the driver keeps the last 1500 characters of the output: the summary of every leg goes last and fits there"""
    sys.path.insert(0, ROOT)
    import bench
    leg = {"ms_per_step": 1.2345678, "solves_per_s": 1234.5678, "mparticles_per_s": 123.45678,
           "latency_p50_s": 1.23456, "latency_p99_s": 2.3456}
    line = {"value": 265.123456, "e2e": {"value": 244.6789}, "roofline": {"frac": 0.6678901},
            "build_hbm": {"gbs": 1900.12345, "peak_gbs": 6456.0},
            "phase_ms": {k: 12.3456789 for k in ("sort", "tree", "upsweep", "traverse", "total")},
            "interactions": {"p2p_per_body": 3788.123456, "m2p_per_body": 1291.987654},
            "accuracy": {"err_p99_1st_pct": 7.3456789e-4, "err_max": 1.23456e-2},
            "accuracy_matched": {"theta": 0.43, "value": 197.123456, "err_p99_1st_pct": 4.7123e-4},
            "ensemble": {"batched": leg, "plain_loop": leg, "speedup_solves_per_s": 9.3456},
            "served": {"served": leg, "plain": leg, "speedup_solves_per_s": 1.3345},
            "plummer_2e24": {"fixed_groups": {"mparticles_per_s": 161.7123, "err_p99_1st_pct": 4.47e-4,
                                              "err_max": 1.549e-3}},
            "precision": {"summary": {"note": "hernquist: 1st-pct rel err; periodic: p99 err / rms|a|",
                                      "hernquist": {"0.3": 2.1123e-4, "0.5": 1.9123e-3, "0.7": 6.9123e-3},
                                      "periodic": {"0.3": 1.7123e-3, "0.5": 2.2123e-3, "0.7": 6.4123e-3}}}}
    line["summary"] = bench.summarize(line)
    text = json.dumps(line)
    assert list(line)[-1] == "summary"
    tail = json.dumps({"summary": line["summary"]})
    assert len(tail) < 1400, len(tail)
    assert text.endswith(tail[1:])
    s = line["summary"]
    assert s["acc_theta_0.5"]["p99"] == 7.346e-4 and s["acc_matched"]["theta"] == 0.43
    assert s["acc_matched"]["mps"] == 197.1
    assert s["ensemble"]["x"] == 9.346 and s["served"]["served_latency_p99_s"] == 2.346


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_summary_reads_samples_and_reasons():
    """the clock record: median SM clock, the maximum, and every throttle reason seen active in any sample, from
    NVML samples and from nvidia-smi lines alike"""
    b = _bench_module()
    c = b.ClockSampler("GPU-unused")
    c.samples = [(1965.0, 1965.0, set()), (1950.0, 1965.0, {"sw_power_cap"})]
    c.lines = ["1800, 1965, 700.5, Active, Active, Not Active, Not Active, Not Active", "garbage"]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert b.ClockSampler("GPU-unused").summary()["samples"] == 0
