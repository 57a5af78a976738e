"""bench.py's reference arm on the CPU (no GPU needed): one JSON line with the
fields of the bench contract, timing the oracle restatement of TAN's CPU path
on the workload's shape; under torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "6",
                          "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout


def test_reference_arm_prints_one_contract_line():
    lines = [ln for ln in _run({"RANK": "0", "WORLD_SIZE": "1"}).splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GSamples/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 6 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["ms_per_step"] > 0 and d["scaling"] == "weak" and d["dtype"] == "f32" and d["data"] == "synthetic"
    assert d["vs_baseline"] is None and "workload" in d["config"]
    assert d["config"]["channels"] == 64 and d["config"]["block"] == 512 and d["config"]["ir_length"] == 65536
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GSamples/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    assert not [ln for ln in _run({"RANK": "1", "WORLD_SIZE": "2"}).splitlines() if ln.startswith("{")]


def test_reference_arm_rank_zero_reports_the_world_size():
    lines = [ln for ln in _run({"RANK": "0", "WORLD_SIZE": "2"}).splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and json.loads(lines[0])["n_gpus"] == 2
