"""bench.py's output contract, checked on the CPU through its reference arm
(the oracle port timed on the host): one JSON line with the keys, types and
values the contract fixes, and, under torchrun with two ranks, that line from
rank 0 only with every rank exiting 0."""

import json
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(cmd, timeout=300):
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", "4")
    return subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=timeout, env=env)


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.strip().startswith("{")]


def _check_line(d):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert abs(d["ms_per_step"] - 1000.0 / d["value"]) < 1e-6 * d["ms_per_step"]
    assert d["scaling"] in ("weak", "strong") and d["vs_baseline"] is None
    assert d["dtype"] == "f64" and d["data"] == "synthetic" and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_json_line():
    # 64^3 keeps the whole-step timing of the oracle port to seconds here
    r = _run([sys.executable, "bench.py", "--impl", "reference", "--n", "64", "--steps", "1",
              "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_torchrun_rank0_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--size", "64", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    r = _run(cmd)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0


@pytest.mark.gpu
def test_gpu_arm_json_line():
    r = _run([sys.executable, "bench.py", "--n", "64", "--steps", "3", "--warmup", "3",
              "--e2e-steps", "2", "--mixed-error-steps", "2", "--no-ensemble", "--no-adjoint",
              "--no-schemes"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["value"] > 0 and d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert abs(d["ms_per_step"] * d["value"] - 1000.0) < 1e-6 * 1000.0
    rl = d["roofline"]
    assert rl["bound"] in ("hbm", "tensor") and rl["unit"] in ("GB/s", "TFLOP/s")
    assert rl["achieved"] > 0 and rl["peak"] > 0 and abs(rl["frac"] - rl["achieved"] / rl["peak"]) < 1e-12
    assert rl["fp64_pipe"]["peak"] > 0 and 0 < rl["fp64_pipe"]["frac"]
    cb = d["cpu_baseline"]
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] in ("port", "reference")
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    assert d["mixed"]["value"] > 0 and d["mixed"]["rel_linf_err_vs_fp64"] < 1e-4
    oo = d["other_order"]
    assert oo["order"] == 4 and oo["value"] > 0 and oo["max_div"] < 1e-11
    ms = d["mixed_summary"]
    assert ms == d["mixed_form"] and list(d)[-1] == "mixed_form"
    assert abs(ms["vs_fp64_steps_per_s"] - d["mixed"]["value"] / d["value"]) < 1e-12
    # the reference arm states the same workload: identical config objects
    r = _run([sys.executable, "bench.py", "--impl", "reference", "--n", "64", "--steps", "1",
              "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    assert _json_lines(r.stdout)[0]["config"] == d["config"]
