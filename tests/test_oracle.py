"""The CPU oracle (oracle/pds_oracle.c) against known answers of the reference's splat.

The reference ships no tests or golden vectors for this path; these are the self-derived
known answers (kernel mass, the value at a pixel corner, the reference's integer quirks,
finite differences in FP64), plus fixtures produced by the reference extension itself under
tests/golden/ (test_golden.py).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

THREE_OVER_PI = 3.0 / math.pi


def one_photon(px, py, s1, s2, theta, W, H, e=1.0, ch=0):
    """Splat inputs for one photon at pixel position (px, py) with semi-axes s1, s2 px."""
    c, s = math.cos(theta), math.sin(theta)
    M = np.zeros((2, 3, 1))
    M[0, 0, 0] = c / s1 * W / 2
    M[0, 1, 0] = s / s1 * H / 2
    M[1, 0, 0] = -s / s2 * W / 2
    M[1, 1, 0] = c / s2 * H / 2
    xp = np.array([[2 * px / W - 1], [2 * py / H - 1]])
    return (np.array([e]), xp, M, np.array([[ch]], dtype=np.int64),
            np.array([2 * max(s1, s2) / W]))


def test_value_at_corner_is_three_over_pi():
    E, X, M, C, R = one_photon(20, 30, 2.0, 2.0, 0.0, 64, 64, e=1.7)
    img = O.forward(E, X, M, C, R, (1, 64, 64), 20)
    assert img[0, 30, 20] == pytest.approx(1.7 * THREE_OVER_PI, rel=1e-14)


@pytest.mark.parametrize("s1,s2,theta", [(8.0, 8.0, 0.0), (9.0, 5.5, 0.7), (12.0, 6.0, 2.1)])
def test_mass_is_energy_times_area_scale(s1, s2, theta):
    # K integrates to 1 over the unit disk; in pixels the support is the s1 x s2 ellipse
    E, X, M, C, R = one_photon(64.3, 60.8, s1, s2, theta, 128, 128, e=2.0)
    img = O.forward(E, X, M, C, R, (1, 128, 128), 20)
    assert img.sum() == pytest.approx(2.0 * s1 * s2, rel=1e-2)


def test_gm_column2_is_zero_and_ge_is_kernel_sum():
    E, X, M, C, R = one_photon(20.4, 30.7, 3.0, 2.0, 0.3, 64, 64, e=1.3)
    img = O.forward(E, X, M, C, R, (1, 64, 64), 20)
    gE, gX, gM = O.backward(np.ones((1, 64, 64)), E, X, M, C, R, 20)
    assert np.all(gM[:, 2] == 0)
    assert gE[0] * 1.3 == pytest.approx(img.sum(), rel=1e-12)


def _loss_and_grads(G, E, X, M, C, R, shape, mpr):
    img = O.forward(E, X, M, C, R, shape, mpr)
    return float((img * G).sum()), O.backward(G, E, X, M, C, R, mpr)


def test_backward_matches_central_differences_fp64():
    rng = np.random.default_rng(3)
    W = H = 96
    G = rng.standard_normal((1, H, W))
    # photons whose ellipse is well inside the box (no truncation under small shifts)
    E, X, M, C, R = one_photon(40.37, 51.61, 4.2, 2.9, 0.4, W, H, e=0.9)
    R = R * 1.5  # box wider than the support
    _, (gE, gX, gM) = _loss_and_grads(G, E, X, M, C, R, (1, H, W), 20)
    h = 1e-7
    def fd(arr, idx):
        a = arr.copy(); a[idx] += h
        lp = float((O.forward(*(a if arr is v else v for v in (E, X, M, C, R)), (1, H, W), 20) * G).sum())
        a = arr.copy(); a[idx] -= h
        lm = float((O.forward(*(a if arr is v else v for v in (E, X, M, C, R)), (1, H, W), 20) * G).sum())
        return (lp - lm) / (2 * h)
    assert fd(E, (0,)) == pytest.approx(gE[0], rel=1e-6)
    for k in range(2):
        assert fd(X, (k, 0)) == pytest.approx(gX[k, 0], rel=1e-5, abs=1e-6 * abs(gX).max())
    for r in range(2):
        for c in range(2):
            assert fd(M, (r, c, 0)) == pytest.approx(gM[r, c, 0], rel=1e-5, abs=1e-6 * abs(gM).max())


def test_channel_out_of_range_is_skipped():
    E, X, M, C, R = one_photon(20, 20, 2.0, 2.0, 0.0, 32, 32)
    for ch in (1, 5, -1):
        img = O.forward(E, X, M, np.array([[ch]]), R, (1, 32, 32), 20)
        assert not img.any()
        gE, gX, gM = O.backward(np.ones((1, 32, 32)), E, X, M, np.array([[ch]]), R, 20)
        assert not gE.any() and not gX.any() and not gM.any()


def test_coord_to_pixel_truncates_toward_zero():
    # photon half a pixel left of the image: (0.5 x + 0.5) W = -0.5 -> int32 -> 0, not -1
    W = H = 32
    E, X, M, C, R = one_photon(-0.5, 16.0, 3.0, 3.0, 0.0, W, H)
    f5, box = O.footprints(X, C, R, (1, H, W), 20)
    assert f5[0, 0] == 0 and f5[0, 2] == 3
    img = O.forward(E, X, M, C, R, (1, H, W), 20)
    # box columns [0, 3] are visited; with floor the centre would be -1 and column 3 skipped
    assert img[0, 16, 2] > 0
    assert box[0] == 4 * 7


def test_max_pixel_radius_truncates_the_box():
    E, X, M, C, R = one_photon(32.2, 32.6, 6.0, 6.0, 0.0, 64, 64)
    img = O.forward(E, X, M, C, R, (1, 64, 64), 2)
    ys, xs = np.nonzero(img[0])
    assert xs.min() >= 30 and xs.max() <= 34 and ys.min() >= 30 and ys.max() <= 34


def test_ellipse_quirk_on_small_images():
    # the :93 test compares offsets against the image half-size, not the footprint
    W = H = 8
    E, X, M, C, R = one_photon(4.1, 4.2, 20.0, 20.0, 0.0, W, H)
    f5, _ = O.footprints(X, C, R, (1, H, W), 20)
    assert f5[0, 4] == 0  # ellipse test not passed by the whole box
    img = O.forward(E, X, M, C, R, (1, H, W), 20)
    # offset (4, 1) from the centre pixel (4, 4): 16/16 + 1/16 > 1 -> never visited
    assert img[0, 5, 0] == 0 and img[0, 4, 0] > 0 and img[0, 5, 1] > 0


def test_negative_energy_deposits_nothing_but_has_gradient():
    E, X, M, C, R = one_photon(20.3, 20.6, 3.0, 3.0, 0.0, 48, 48, e=-1.0)
    assert not O.forward(E, X, M, C, R, (1, 48, 48), 20).any()
    gE, _, _ = O.backward(np.ones((1, 48, 48)), E, X, M, C, R, 20)
    assert gE[0] > 0


def test_reference_nan_at_zero_radius_and_fp64_limit():
    E, X, M, C, R = one_photon(20, 30, 2.0, 2.0, 0.0, 64, 64)
    G = np.ones((1, 64, 64))
    _, gX32, _ = O.backward(G, E, X, M, C, R, 20, mode="ref32")
    gE, gX, gM = O.backward(G, E, X, M, C, R, 20, mode="fp64")
    assert np.isnan(gX32).all()
    assert np.isfinite(gX).all() and np.isfinite(gM).all()
    assert abs(gX).max() < 1e-9  # symmetric footprint on a constant gradient


def test_photon_off_image_touches_nothing():
    E, X, M, C, R = one_photon(-10.0, 5.0, 2.0, 2.0, 0.0, 32, 32)
    assert not O.forward(E, X, M, C, R, (1, 32, 32), 20).any()


def test_ref32_and_fp64_agree_to_float_precision():
    rng = np.random.default_rng(0)
    W = H = 128
    n = 2000
    pos = rng.uniform(0, W, (2, n))
    s1 = np.exp(rng.uniform(np.log(0.5), np.log(4), n))
    s2 = np.exp(rng.uniform(np.log(0.5), np.log(4), n))
    th = rng.uniform(0, np.pi, n)
    M = np.zeros((2, 3, n), np.float32)
    M[0, 0] = np.cos(th) / s1 * W / 2; M[0, 1] = np.sin(th) / s1 * H / 2
    M[1, 0] = -np.sin(th) / s2 * W / 2; M[1, 1] = np.cos(th) / s2 * H / 2
    X = (2 * pos / W - 1).astype(np.float32)
    E = rng.uniform(0.5, 1, n).astype(np.float32)
    R = (2 * np.maximum(s1, s2) / W).astype(np.float32)
    C = np.zeros((1, n), np.int64)
    a = O.forward(E, X, M, C, R, (1, H, W), 20, mode="fp64")
    b = O.forward(E, X, M, C, R, (1, H, W), 20, mode="ref32")
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-4



def test_philox_known_answers():
    """The numpy Philox4x32-10 (checker of the device photon source) against the published
    known-answer vectors of the algorithm."""
    from oracle import philox as P
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in cases:
        got = P.philox4x32_10([np.array([w], dtype=np.uint64) for w in ctr], key)[:, 0]
        assert [int(v) for v in got] == list(want)


def test_photon_source_restatement_stays_in_texels():
    from oracle import philox as P
    px, py = P.photon_source(5, 7, 3, 0.25, seed=99, offset=4)
    assert px.shape == (105,) and px.dtype == np.float32
    t = np.arange(105) % 35  # sample-major: photon i in texel i % (rows * cols)
    assert np.all(np.abs(px / 0.25 - (t % 7 - 3.0)) <= 0.5)
    assert np.all(np.abs(py / 0.25 - (t // 7 - 2.0)) <= 0.5)
