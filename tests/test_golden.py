"""Pins the CPU oracle on outputs of the reference extension itself.

The fixtures in tests/golden/ were produced by ``tests/golden/make_golden.py``, which runs
the reference's unmodified ``pds_forward`` / ``pds_backward`` (built from its sources by
``oracle/build_ref.py``) on a GPU in float64 and float32. The FP64 oracle must reproduce the
reference's float64 results to rounding (the only differences are the order of the
reference's atomic adds and nvcc's multiply-add contraction); the REF32 mode must reproduce
its float32 results to float rounding, including the NaN gradients of a photon sitting
exactly on a pixel corner.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
# the splat fixtures (refraction_ref.npz holds the refraction chain's, test_refraction_golden.py)
FIXTURES = sorted(f for f in glob.glob(os.path.join(HERE, "golden", "*.npz"))
                  if not os.path.basename(f).startswith("refraction"))


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a, np.float64) - b) / (nb if nb > 0 else 1.0)


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def valid_channel(f):
    c = f["C"].reshape(-1)
    return (c >= 0) & (c < int(f["shape"][0]))


def test_fixtures_present():
    assert len(FIXTURES) >= 6, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_fp64_matches_reference_float64(path):
    f = load(path)
    shape, mpr = tuple(int(v) for v in f["shape"]), int(f["mpr"])
    img = O.forward(f["E"], f["X"], f["M"], f["C"], f["R"], shape, mpr, mode="fp64")
    assert rel_l2(img, f["img_f64"]) < 1e-12
    gE, gX, gM = O.backward(f["G"].astype(np.float64), f["E"], f["X"], f["M"], f["C"], f["R"],
                            mpr, mode="fp64")
    ok = valid_channel(f)
    # the reference's 0/0 at r = 0 poisons a photon's dL/dx and dL/dM; compare the others
    finite = ok & np.isfinite(f["gX_f64"]).all(0) & np.isfinite(f["gM_f64"]).all((0, 1))
    assert rel_l2(gE[ok], f["gE_f64"][ok]) < 1e-12
    assert rel_l2(gX[:, finite], f["gX_f64"][:, finite]) < 1e-10
    assert rel_l2(gM[:, :, finite], f["gM_f64"][:, :, finite]) < 1e-10
    assert np.isfinite(gX).all() and np.isfinite(gM).all()


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_ref32_matches_reference_float32(path):
    f = load(path)
    shape, mpr = tuple(int(v) for v in f["shape"]), int(f["mpr"])
    img = O.forward(f["E"], f["X"], f["M"], f["C"], f["R"], shape, mpr, mode="ref32")
    assert rel_l2(img, f["img_f32"]) < 1e-5
    gE, gX, gM = O.backward(f["G"].astype(np.float64), f["E"], f["X"], f["M"], f["C"], f["R"],
                            mpr, mode="ref32")
    ok = valid_channel(f)
    # NaN pattern (photons on a pixel corner) is reproduced exactly
    assert np.array_equal(np.isnan(gX[:, ok]), np.isnan(f["gX_f32"][:, ok]))
    finite = ok & np.isfinite(f["gX_f32"]).all(0) & np.isfinite(f["gM_f32"]).all((0, 1))
    assert rel_l2(gE[ok], f["gE_f32"][ok]) < 1e-4
    assert rel_l2(gX[:, finite], f["gX_f32"][:, finite]) < 1e-4
    assert rel_l2(gM[:, :, finite], f["gM_f32"][:, :, finite]) < 1e-4


def test_corner_fixture_has_the_reference_nan():
    p = os.path.join(HERE, "golden", "corner_32.npz")
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    f = load(p)
    assert np.isnan(f["gX_f32"][:, 0]).all() and np.isnan(f["gX_f64"][:, 0]).all()
    assert np.isfinite(f["gX_f32"][:, 1:]).all()
