"""The JSON line of ``bench.py --impl reference`` (the CPU reference arm), run here on the CPU.

The reference arm times the reference's splat formula (the float32-order CPU port) on a
bounded photon sample per step of the benchmark workload; its line carries the same metric,
unit and workload as the CUDA arm plus ``impl``, ``cpu_baseline`` and a host-only ``e2e``.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run(
        [sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "0",
         "--ref-sample", "32768"],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    r = json.loads(lines[0])
    assert r["impl"] == "reference"
    assert r["metric"] == "photon fwd+bwd splats/s" and r["unit"] == "photons/s"
    assert r["higher_is_better"] is True and r["n_gpus"] == 1
    assert r["steps"] == 2 and r["warmup"] == 0
    assert r["value"] > 0 and r["ms_per_step"] > 0
    assert r["config"]["workload"].startswith("batch64")
    assert r["config"]["sample_photons_per_step"] == 32768
    cb = r["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == r["value"] and cb["unit"] == r["unit"]
    e2e = r["e2e"]
    assert e2e["value"] == r["value"] and e2e["unit"] == r["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
