"""bench.py end to end on a small mesh: every leg of the default JSON line
(RHS, end-to-end copies, RK and IMEX time steps, the pressure-solve
comparison, the CPU baseline) runs, and the line carries every key of the
bench line format.  The legs are those of the default run, at sizes that take seconds."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu


def test_default_line_all_legs_small():
    cmd = [sys.executable, "bench.py", "--nelem1d", "8", "--steps", "3", "--warmup", "3", "--p-nelem1d", "4",
           "--p-harvest", "3", "--p-compare", "3", "--p-train", "2", "--p-self", "1", "--p-finetune", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [l for l in p.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks", "cpu_baseline",
              "time_step", "imex_step", "pressure_solve"):
        assert k in d, k
    assert d["value"] > 0 and d["roofline"]["frac"] > 0 and d["e2e"]["value"] > 0
    assert d["time_step"]["ms_per_step"] > 0 and d["imex_step"]["ms_per_step"] > 0
    ps = d["pressure_solve"]
    assert ps["learned"]["max_true_residual"] < 1e-8 and ps["jacobi"]["max_true_residual"] < 1e-8
    assert ps["jacobi_extrapolated_guess"] is not None and ps["speedup_wall"] > 0
