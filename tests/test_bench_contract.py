"""bench.py's reference arm on the CPU: the JSON line it prints (the CPU
implementation of the path, timed on the host's cores) and its behaviour
under torchrun, on a small workload.  The B200 arm needs a GPU and is run by
the GPU runs."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                       env=e, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def test_reference_arm_line():
    out = _bench("--impl", "reference", "--steps", "2", "--warmup", "3", "--n-obs", "4096",
                 "--cpu-seconds", "0.5")
    line = json.loads(out.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["steps"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and line["unit"] == "chain-obs/s"
    assert line["config"]["n_obs"] == 4096 and "2^12" in line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_nothing():
    # under torchrun only rank 0 runs and prints the reference line
    out = _bench("--impl", "reference", "--steps", "1", "--warmup", "3", "--n-obs", "1024",
                 env={"RANK": "1", "WORLD_SIZE": "2"})
    assert out.strip() == ""
