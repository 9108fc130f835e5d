"""bench.py's reference arm (`--impl reference`): the reference's own CPU sigma (oracle/_ref/ref_bench,
sbd::mult of tpb/mult.h:625-881) timed per step on a bra-row block of the whole problem (every
connection of the block's rows), printed as one JSON line with the keys of the benchmark contract.
Runs on the CPU, here on the 24-orbital workload with 1-second blocks; under torchrun with two ranks
(gloo), rank 0 alone prints the line and the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
ARGS = ["--impl", "reference", "--workload", "sci24", "--steps", "1", "--warmup", "0", "--cpu-step-seconds", "1"]
needs_ref = pytest.mark.skipif(not os.path.exists(REF_BENCH), reason="oracle/_ref not built")


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check_line(d, n_gpus):
    assert d["impl"] == "reference"
    assert d["unit"] == "GDets/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["n_gpus"] == n_gpus and d["steps"] == 1 and d["warmup"] == 0 and d["ms_per_step"] > 0
    assert d["metric"].startswith("sigma GDets/s")
    assert d["config"]["workload"].startswith("sci24: norb=24")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GDets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the sample covers the whole problem's connections: blocks of whole alpha rows x all beta strings
    assert d["config"]["determinants"] == 4000 * 4000
    b = d["blocks"]
    assert 1 <= b["rows"] <= 4000 and len(b["block_s"]) == d["steps"] + d["warmup"] and b["fixed_s"] >= 0


@needs_ref
def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py"] + ARGS, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 1)


@needs_ref
def test_reference_arm_two_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--gpus", "2"] + ARGS
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 2)
