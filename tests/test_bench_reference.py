"""The reference arm of bench.py runs on the host alone: its JSON line keeps
the contract (metric, unit, impl, cpu_baseline, e2e with no transfers) on a
small grid, so the driver's round-end run of that arm can be trusted."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.isdir(os.path.join(ROOT, "oracle", "_ref")), reason="reference not built here")
def test_reference_arm_json_line():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--nx", "16", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    assert line["impl"] == "reference" and line["unit"] == "ms" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["outer_iters"] >= 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 2 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
