"""The bench's own arm on the small channel: one JSON line with the keys the
contract names (throughput, device and end-to-end, roofline of the far
field, per-stage HBM figures, clocks, launch count)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_bench_line_has_the_contract_keys(cuda):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", "channel2d", "--steps", "3",
                          "--warmup", "3", "--no-cpu-baseline", "--no-vs-bs", "--no-extras"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    r = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "e2e",
              "stages_ms", "stage_roofline", "vvpe_applied_fraction"):
        assert k in r, k
    assert r["n_gpus"] == 1 and r["steps"] == 3 and r["warmup"] >= 3 and r["value"] > 0
    assert r["gpu_launches"] > 0 and "workload" in r["config"]
    rf = r["roofline"]
    assert rf["bound"] in ("fp32", "hbm", "tensor") and 0 < rf["frac"] < 1.5 and rf["peak"] > 0
    e = r["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert set(r["stage_roofline"]["stages"]) <= {"grid", "dfsph", "dimcv_sweeps"}
    a = r["vvpe_applied_fraction"]
    assert 0.0 < a["fraction"] <= 1.0 and a["fluid_rows"] > 0
