"""FP64 restatement of the point light's photon directions. TEST INFRASTRUCTURE ONLY: the
checker of ``pds_point_light_source_f32``; the product never imports it. Pinned to the
reference's ``compute_point_light_dirs`` by ``tests/golden/refraction_ref.npz``.

Restates ``model/caustics.py:26-70`` with ``model/utils.py``'s ``slerp``,
``compute_orthonormal_basis`` (Frisvad 2012) and ``subtended_angle`` (Van Oosterom and
Strackee 1983): directions are the bilinear slerp of the four corner directions of the
rectangle [xmin, xmax] x [ymin, ymax] at z = plane_z, their differentials the orthonormal basis
scaled by 2 smoothing sqrt(omega / (pi N)).
"""
import math

import numpy as np

from oracle import philox

__all__ = ["slerp", "onb", "subtended_angle", "point_light", "philox_coeffs"]


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def slerp(p0, p1, t):
    """[..., 3] vectors, t [..., 1]."""
    w = np.arccos(np.clip((p0 * p1).sum(-1, keepdims=True), -1.0, 1.0))
    return (np.sin((1 - t) * w) * p0 + np.sin(t * w) * p1) / np.sin(w)


def onb(n, eps=1e-5):
    """Frisvad's orthonormal basis (b1, b2) of unit vectors n [N, 3]."""
    nx, ny, nz = n[:, 0], n[:, 1], n[:, 2]
    sing = nz < -1 + eps
    a = 1 / np.where(sing, 1.0, 1 + nz)
    b = -nx * ny * a
    b1 = np.stack((1 - a * nx ** 2, b, -nx), -1)
    b2 = np.stack((b, 1 - a * ny ** 2, -ny), -1)
    b1[sing] = (0.0, -1.0, 0.0)
    b2[sing] = (-1.0, 0.0, 0.0)
    return b1, b2


def _tri(o, v0, v1, v2):
    d0, d1, d2 = v0 - o, v1 - o, v2 - o
    n0, n1, n2 = (np.linalg.norm(d) for d in (d0, d1, d2))
    num = float(np.dot(d0, np.cross(d2, d1)))
    den = n0 * n1 * n2 + n0 * np.dot(d1, d2) + n1 * np.dot(d0, d2) + n2 * np.dot(d0, d1)
    a = 0.0 if (num == 0 and den == 0) else 2 * math.atan2(num, den)
    return max(a, 0.0)


def subtended_angle(o, xmin, ymin, xmax, ymax, z):
    p00, p10 = np.array([xmin, ymin, z]), np.array([xmax, ymin, z])
    p01, p11 = np.array([xmin, ymax, z]), np.array([xmax, ymax, z])
    return _tri(o, p00, p10, p01) + _tri(o, p01, p10, p11)


def point_light(o, rect, plane_z, u0, u1, smoothing, energy, simulations, inner, wavelengths=1):
    """-> direction, dtheta, dphi ([N, 3], directions repeated per wavelength), flux [N]."""
    o = np.asarray(o, np.float64)
    xmin, ymin, xmax, ymax = rect
    corners = [np.array([x, y, plane_z]) for x, y in ((xmin, ymin), (xmax, ymin),
                                                       (xmin, ymax), (xmax, ymax))]
    c00, c10, c01, c11 = (_unit(c - o) for c in corners)
    u0 = np.asarray(u0, np.float64)[:, None]
    u1 = np.asarray(u1, np.float64)[:, None]
    lower = slerp(c00[None], c10[None], u0)
    upper = slerp(c01[None], c11[None], u0)
    d = slerp(lower, upper, u1)
    b1, b2 = onb(d)
    n_dir = d.shape[0]
    omega = subtended_angle(o, xmin, ymin, xmax, ymax, plane_z)
    scale = 2 * smoothing * math.sqrt(omega / (math.pi * n_dir * simulations * wavelengths))
    rep = lambda a: np.repeat(a, wavelengths, axis=0)  # noqa: E731
    flux = np.full(n_dir * wavelengths, energy / (simulations * inner))
    return rep(d), rep(scale * b1), rep(scale * b2), flux


def philox_coeffs(n_dir, seed, offset):
    """(u0, u1) of the device source: two directions per Philox block, top 24 bits."""
    pairs = (n_dir + 1) // 2
    ctr = np.arange(pairs, dtype=np.uint64) + np.uint64(offset)
    words = philox.philox4x32_10([ctr & np.uint64(0xFFFFFFFF), ctr >> np.uint64(32),
                                  np.zeros(pairs, np.uint64), np.zeros(pairs, np.uint64)],
                                 (seed & 0xFFFFFFFF, seed >> 32))
    unit = lambda w: (w >> np.uint64(8)).astype(np.float64) / 16777216.0  # noqa: E731
    u0 = np.stack((unit(words[0]), unit(words[2])), 1).reshape(-1)[:n_dir]
    u1 = np.stack((unit(words[1]), unit(words[3])), 1).reshape(-1)[:n_dir]
    return u0, u1
