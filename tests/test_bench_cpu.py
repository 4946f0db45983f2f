"""bench.py's reference arm (bounded samples of the headline solve on the
host cores: the oracle's H|psi> and subspace products, no GPU) prints one
JSON line with the keys of the benchmark contract, and its value is the
work it completed inside its own clock: the solve fraction of a step over
the step's measured time, consistent with ms_per_step."""

import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0.0 and line["higher_is_better"] is True
    assert line["config"]["workload"] == "si64_scf_gamma_30ry"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    frac = line["solve_fraction_per_step"]
    assert 0.0 < frac < 1.0
    assert abs(line["value"] * line["ms_per_step"] * 1e-3 - frac) <= 1e-9 * frac
