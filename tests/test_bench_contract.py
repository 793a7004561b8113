"""bench.py's reference arm (``--impl reference``): rank 0 prints exactly one
JSON line in the benchmark's contract, timing the oracle's CPU restatement of
the reference's classic path on the host cores.  Needs no GPU."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup = 1, 0

    assert bench.run_reference(A(), 0, 1) == 0
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "GB/s" and d["higher_is_better"] is True
    for key in ("value", "n_gpus", "steps", "warmup", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e", "data_gibs"):
        assert key in d, key
    assert d["value"] > 0 and d["data_gibs"] > 0
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
