"""``bench.py`` on the GPU: one short run of the CUDA arm and the keys of its JSON line.

Runs the 2^20-photon 512^2 workload for three timed steps (library default configuration, a
short CPU-baseline sample) and checks that the line carries the metric, the device roofline,
the end-to-end number with its copied bytes, the launch count, the sampled clocks, the CPU
baseline, the step's error against the FP64 oracle, the whole-step roofline and the reference
CUDA extension's run on the same workload.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_carries_every_key(cuda):
    out = subprocess.run(
        [sys.executable, "bench.py", "--workload", "uniform1m", "--steps", "3", "--warmup", "3",
         "--no-autotune", "--cpu-seconds", "0.5"],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout + out.stderr
    r = json.loads(lines[0])
    assert r["metric"] == "photon fwd+bwd splats/s" and r["unit"] == "photons/s"
    assert r["n_gpus"] == 1 and r["steps"] == 3 and r["warmup"] == 3
    assert r["value"] > 0 and r["ms_per_step"] > 0 and r["higher_is_better"] is True
    assert r["scaling"] == "weak" and r["dtype"] == "f32"
    assert r["config"]["workload"].startswith("uniform1m")
    rl = r["roofline"]
    assert rl["bound"] in ("hbm", "tensor") and rl["unit"] == "GB/s"
    assert rl["achieved"] > 0 and rl["peak"] > 0
    assert abs(rl["frac"] - rl["achieved"] / rl["peak"]) < 1e-9
    e2e = r["e2e"]
    assert e2e["unit"] == r["unit"] and 0 < e2e["value"]
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert r["gpu_launches"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(r["clocks"])
    cb = r["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] > 0
    # per-result error of the timed step against the FP64 oracle, within the stated tolerances
    pv = r["parity_vs_oracle"]
    assert pv["image"] <= 1e-5 and pv["photons"] == 2 ** 20
    assert max(pv["grad_Ep"], pv["grad_xp"], pv["grad_Mp"]) <= 1e-4
    # the whole step against the roofline
    rs = r["roofline_step"]
    assert rs["algorithmic_bytes"] == 2 ** 20 * 116 + 512 * 512 * 8
    assert abs(rs["frac"] - rs["achieved"] / rs["peak"]) < 1e-9
    # the reference's own CUDA extension on the same workload (when it is built)
    rg = r["reference_gpu"]
    assert "unavailable" in rg or (rg["value"] > 0 and rg["ours_over_reference_gpu"] > 0)


def test_plate_batch_iteration_runs_batched_and_plain(cuda):
    """The batched-vs-plain Landweber iteration with refraction that the benchmark line carries
    (64 simulations with their own tilt, wavelength, photon count and image size)."""
    import torch
    sys.path.insert(0, ROOT)
    import bench
    r = bench.run_plate_batch(None, torch.device("cuda:0"), 2, 1)
    assert r["simulations"] == 64 and r["photons_per_iteration"] > 2 ** 24
    assert r["batched_it_per_s"] > 0 and r["plain_it_per_s"] > 0
    assert r["batched_over_plain"] > 1.0
