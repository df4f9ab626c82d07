"""bench.py's reference arm (Teide's own CPU engine, oracle/_ref) prints the
one-line JSON contract: the same metric, unit and workload names as the
device arm, a cpu_baseline block describing the run, and an e2e block with no
host<->device bytes.  Runs on the CPU at 2% of each workload's size in a few seconds."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libteide_ref.so")


@pytest.mark.parametrize("workload", ["join_group", "group_sort"])
def test_reference_arm_prints_contract_line(workload):
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libteide_ref.so not built")
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", workload,
                        "--steps", "1", "--warmup", "3", "--scale", "0.02"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout[-2000:]
    r = json.loads(lines[0])
    assert r["impl"] == "reference"
    assert r["config"]["workload"] == workload and r["config"]["scale"] == 0.02
    # the same config object the device arm prints for this workload and size
    sys.path.insert(0, ROOT)
    import bench
    rows, alg, _ = bench.workload_rows(workload, bench.workload_inputs_shape(workload, 0.02))
    assert r["config"] == json.loads(json.dumps(bench.bench_config(workload, rows, alg, 1, 0.02)))
    assert r["unit"] == "rows/s" and r["higher_is_better"] is True
    assert r["value"] > 0 and r["steps"] == 1 and r["warmup"] == 3 and r["n_gpus"] == 1
    cb = r["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == r["value"] and cb["sample"]
    assert r["e2e"] == {"value": r["value"], "unit": r["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
