"""bench.py's output contract, on the CPU: the reference arm (`--impl reference`) runs the
oracle only, so it runs here.  One JSON line carries the metric, the whole-job value, the timing
keys, the workload's config, `cpu_baseline` and an `e2e` with no host-device bytes; under
torchrun with two ranks only rank 0 prints it and the other rank exits 0 without work; and the
arm's process maps the oracle's library but never this library's."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--impl", "reference", "--scale", "13", "--batch", "500", "--steps", "3", "--warmup", "3"]
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check_line(d, gpus):
    assert KEYS <= set(d), sorted(KEYS - set(d))
    assert d["impl"] == "reference" and d["n_gpus"] == gpus
    assert (d["steps"], d["warmup"]) == (3, 3)
    assert d["unit"] == "changed edges/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    c = d["config"]
    assert c["workload"] == "rmat-s13-ef16-w1000-batch500" and c["batch_changes"] == 500
    assert c["l2"].startswith("inputs smaller than L2")  # a small configuration says so
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "changed edges/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_prints_one_contract_line():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + SMALL, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _lines(p.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 1)


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--gpus", "2"] + SMALL
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    if p.returncode != 0 and "address already in use" in (p.stderr + p.stdout).lower():
        pytest.skip("rendezvous port taken")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _lines(p.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 2)
    assert lines[0]["config"]["parallelism"] == "replicas2"


def test_reference_arm_loads_the_oracle_and_not_this_library():
    probe = ("import runpy, sys\n"
             f"sys.argv = ['bench.py'] + {SMALL!r}\n"
             "runpy.run_path('bench.py', run_name='__main__')\n"
             "maps = open('/proc/self/maps').read()\n"
             "print('MAPS', 'libdyngb200' in maps, 'liboracle' in maps)\n")
    p = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "MAPS False True" in p.stdout, p.stdout[-500:]
