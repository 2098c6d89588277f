"""The reference arm of bench.py on the host (no GPU): `--impl reference`
times the reference's own CPU functions (or the C restatement when the
reference build is absent) single-threaded and as one process per core,
and prints one JSON line with the keys the bench contract asks for."""

import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "halfspace_20x20x10",
                          "--steps", "1", "--warmup", "3", "--cpu-seconds", "2"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "GLL-pt/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "halfspace_20x20x10"
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    # one process per core stepping its own part of the sample beats one thread
    assert d["cpu_baseline"]["single_thread"] > 0
    assert d["value"] >= d["cpu_baseline"]["single_thread"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
