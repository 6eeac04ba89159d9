"""The reference arm of bench.py on CPU: `--impl reference` times the FP64
C++ restatement of the reference's CPU randomized PCA on the host cores and
prints one JSON line with the bench contract's keys; under torchrun only rank 0
prints.  Small sample so the test takes seconds."""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--n-obs", "4000", "--cpu-sample-rows", "4000",
           "--steps", "1", "--warmup", "0"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "ms" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["ms_per_step"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "ms", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["n_obs"] == 4000


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
