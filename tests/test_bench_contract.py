"""bench.py's reference arm (`--impl reference`: the oracle on the host cores)
keeps the JSON-line contract on the CPU: one line with the metric, value,
unit, impl, the run's sizes, the workload config that the GPU arm reports
for the same workload, a cpu_baseline describing the sample, and an e2e with
no host-device copies; under a multi-rank launch only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(extra_env=None, *args):
    env = dict(os.environ)
    env.update(extra_env or {})
    env.setdefault("OMP_NUM_THREADS", "4")
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, cwd=ROOT, timeout=600)


def test_reference_arm_json_line():
    r = run(None, "--workload", "c1_1d_l64", "--steps", "3", "--warmup", "1")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["vs_baseline"] is None
    assert d["steps"] >= 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the same config dict the GPU arm prints for this workload
    sys.path.insert(0, ROOT)
    import bench
    from fastearth3d_b200 import synth

    w = synth.workloads()["c1_1d_l64"]
    assert d["config"] == bench.workload_config(w, d["config"]["n_sub"], 1)


def test_reference_arm_other_ranks_print_nothing():
    r = run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--workload", "c1_1d_l64", "--steps", "2",
            "--warmup", "1")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
