"""bench.py's reference arm without a GPU: the line the benchmark contract
asks for, from the reference's own CPU code (oracle/_ref/ref_harness, built
from the reference's sources by oracle/Makefile), on the small c1 workload;
and the c4 arm's `unavailable` line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def bench_line(*args):
    env = dict(os.environ)
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                         env=env, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout + out.stderr
    return json.loads(lines[0])


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="oracle/_ref/ref_harness not built")
def test_reference_arm_line_on_c1():
    d = bench_line("--impl", "reference", "--workload", "c1", "--steps", "2", "--warmup", "1",
                   "--ref-reps", "1")
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["metric"] and d["unit"] == "edge-visits/s"
    assert d["higher_is_better"] is True
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 2, 1)
    assert d["value"] > 0 and d["ms_per_step"] > 0
    # value = the workload's edge visits per step / the step's time
    visits = d["config"]["edge_visits_per_step"]
    assert abs(d["value"] * d["ms_per_step"] / 1e3 - visits) <= 1e-6 * visits
    assert d["config"]["workload"].startswith("c1")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    p = d["detail"]["protocol"]
    assert p["table_method"] in ("ParGrid", "ParGridPlus", "ParCoreIndex")
    assert p["table_setting"] in ("as_shipped", "thread_limit")


def test_reference_arm_c4_is_unavailable_not_an_error():
    d = bench_line("--impl", "reference", "--workload", "c4", "--steps", "1", "--warmup", "0")
    assert d["impl"] == "reference" and d["unavailable"]


def test_reference_arm_other_ranks_exit_without_work():
    # under torchrun rank 0 alone times the reference; the others print nothing
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2",
               MASTER_ADDR="127.0.0.1", MASTER_PORT="29533")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "c1", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]
