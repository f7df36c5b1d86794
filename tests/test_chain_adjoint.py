"""The refraction backward's reverse-mode sweeps against forward-mode dual numbers, on the
host (no GPU): tests/chain_adjoint_check.cu instantiates the chain templates of
``shapefromcaustics_b200/csrc/pds_chain.cuh`` with dual numbers (seven tangents) and compares
their derivatives with ``plate_chain_adjoint`` and ``point_chain_adjoint`` on 300 seeded
random photons each. Both are float32: relative L2 of the seven derivatives at the median
photon <= 1e-5; the worst photons (nearly singular footprints, where both evaluations lose
digits to cancellation) <= 1e-4 (collimated) and 1e-3 (point light)."""
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    p = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return p if os.path.exists(p) else shutil.which("nvcc")


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_reverse_sweeps_match_dual_numbers(tmp_path):
    exe = str(tmp_path / "chain_adjoint_check")
    subprocess.check_call([_nvcc(), "-std=c++17", "-O2", "-x", "cu",
                           os.path.join(HERE, "chain_adjoint_check.cu"), "-o", exe])
    out = subprocess.check_output([exe], text=True)
    res = {}
    for line in out.splitlines():
        m = re.match(r"(\w+) trials (\d+) median (\S+) worst (\S+)", line)
        if m:
            res[m.group(1)] = (int(m.group(2)), float(m.group(3)), float(m.group(4)))
    assert set(res) == {"collimated", "point"}, out
    for name, worst in (("collimated", 1e-4), ("point", 1e-3)):
        n, med, wst = res[name]
        assert n >= 250, out
        assert med <= 1e-5 and wst <= worst, out
