"""bench.py's reference arm on the host: the reference's own CPU av() on the
m=1024 microbench, one JSON line with the contract's keys (no GPU needed)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liboref_u1.so")):
        pytest.skip("reference build (oracle/_ref) not present")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "3", "--cpu-sample-s", "0.3"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "matvec/s" and d["higher_is_better"] is True
    assert d["metric"].startswith("H_eff matvec/s at m=1024")
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 3
    assert d["config"]["psi_elems"] == 599964 and d["config"]["tasks"] == [190, 190]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "sample" in cb
    assert d["e2e"] == {"value": d["value"], "unit": "matvec/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
