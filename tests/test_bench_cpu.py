"""bench.py's reference arm (the oracle, the C++ restatement of the
reference's SA path, on the host cores) keeps the benchmark's JSON contract
without a GPU: one line with impl, metric, unit, value, the device arm's
config, cpu_baseline and e2e; ranks other than 0 print nothing."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(rank_env):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env.update(rank_env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--reference-sample-s", "0.3"],
                          capture_output=True, text=True, env=env, timeout=300)


def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["unit"] == "pair-integrals/s" and d["higher_is_better"] is True
    assert d["metric"].startswith("E_l assembly pair-integrals/s") and d["value"] > 0 and d["ms_per_step"] > 0
    cfg = d["config"]
    assert cfg["workload"] == "sphere_icosphere3_N1280_L40_GH7" and cfg["pair_integrals_per_step"] == 26_678_800
    # the step time is the measured time of the sampled work, not an extrapolation to a full step
    assert d["ms_per_step"] <= 1e3 * (cb_s := d["cpu_baseline"]["seconds"]) * 1.0001 + 1e-9
    assert d["ms_per_step"] < 60_000 and "sample" in cfg["reference_step"]
    assert cfg["l2"].startswith("output 4.72 GB per step")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
