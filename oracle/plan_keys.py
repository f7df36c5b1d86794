"""CPU restatement of the splat plan's binning keys. TEST INFRASTRUCTURE ONLY: the tests hold
the device plan (``pds_plan_f32`` / ``pds_batch_plan_f32``, read back through
``pds_plan_export``) to it bit for bit; the product never imports it.

The reference has no binning: each of its threads walks one photon's box
(``PyOptix/kernel/photon_differentials.cu:76-110``). The key restated here is this library's:
per photon, its footprint by the reference's integer rules (``:76-87``, via the FP64 oracle's
``footprints``), its clipped box, and

  - ``(n_tiles + 1) << class_bits`` (touches no pixel) when its channel lies outside
    ``[0, C)`` or its clipped box is empty;
  - ``n_tiles << class_bits`` (wide) when ``rx`` or ``ry`` exceeds the apron
    ``min(max_pixel_radius, apron_max)``;
  - otherwise ``(tile << class_bits) | class`` with ``tile = tile_base + (c * tiles_y + ty) *
    tiles_x + tx`` of the centre pixel clamped into the image, and, for the default 6 class
    bits, the row class: 3 bits for the band's rows inside the box and 3 for its width
    (levels 1, 2, 3, 4, 5-6, 7-8, 9-12, 13+), computed in IEEE single precision in the
    order the device uses, class 63 for photons without a band.
"""
import numpy as np

from oracle import oracle as O

__all__ = ["row_level", "row_class", "plan_keys"]

F32 = np.float32


def row_level(v):
    v = np.maximum(np.asarray(v), 1)
    return np.where(v <= 4, v - 1, np.where(v <= 6, 4, np.where(v <= 8, 5, np.where(v <= 12, 6, 7))))


def row_class(m00, m01, m10, m11, dy0, W, H, rx, kxb0, kxb1, kyb0, kyb1):
    """The row class of each photon (float32 arrays; integer box offsets)."""
    with np.errstate(all="ignore"):
        m00, m01, m10, m11, dy0 = (np.asarray(v, F32) for v in (m00, m01, m10, m11, dy0))
        a = m00 * m00 + m10 * m10
        p = m00 * m11
        q = m01 * m10
        det = p - q
        ok = (a > 0) & (a < F32(1e30))
        ok &= np.abs(det) > F32(1e-3) * (np.abs(p) + np.abs(q))
        isx = F32(0.5) * F32(W)
        isy = F32(0.5) * F32(H)
        sa = np.sqrt(a)
        hw = isx / sa
        ey = sa / np.abs(det)
        ok &= (hw <= np.asarray(rx, F32) + F32(1)) & (ey * isy < F32(1e6))
        ky0 = np.ceil((-ey - dy0) * isy)
        ky1 = np.floor((ey - dy0) * isy)
        bw = np.floor(F32(2) * hw)
        ky0 = np.where(ok, ky0, 0).astype(np.int64)
        ky1 = np.where(ok, ky1, 0).astype(np.int64)
        bw = np.where(ok, bw, 0).astype(np.int64) + 2
    rows = np.maximum(np.minimum(ky1, kyb1) - np.maximum(ky0, kyb0) + 1, 0)
    w = np.minimum(bw, np.asarray(kxb1) - np.asarray(kxb0) + 1)
    cls = (row_level(rows) << 3) | row_level(w)
    return np.where(ok, cls, 63).astype(np.int64)


def _corner_offset(p_c, W, x):
    """(2 p_c / W - 1) - x in double, separately rounded, then float32."""
    return ((p_c.astype(np.float64) * (2.0 / float(W)) - 1.0) - x.astype(np.float64)).astype(F32)


def plan_keys(photons, sims, max_pixel_radius, tile=64, apron_max=32, class_bits=6):
    """Keys of every photon. ``photons``: (Ep, xp, Mp, cp, radius) numpy arrays in the
    reference's layouts (float32 values); ``sims``: list of (n_photons, (C, H, W)), photons
    concatenated in that order. -> (keys uint64 [N], n_tiles).

    class_bits 6: the full keys (the row walk's classes, computed with correctly rounded
    operations on the device). Other class_bits: the keys with the class field zero, since the
    band walk's area classes come from the device's approximate reciprocal square root; compare
    ``key >> class_bits`` (simulation, channel and tile, and the two sentinels) for those."""
    if not 1 <= class_bits <= 6:
        raise ValueError("class_bits must be in [1, 6]")
    E, X, M, C, R = photons
    X = np.asarray(X, F32)
    M = np.asarray(M, F32)
    C = np.asarray(C).reshape(-1)
    R = np.asarray(R, F32)
    apron = max(min(int(max_pixel_radius), int(apron_max)), 0)
    n_tiles = sum(c * ((h + tile - 1) // tile) * ((w + tile - 1) // tile)
                  for _, (c, h, w) in sims)
    key_big = n_tiles << class_bits
    key_invalid = (n_tiles + 1) << class_bits
    keys = np.empty(C.shape[0], dtype=np.int64)
    b, tile_base = 0, 0
    for n, (nc, H, W) in sims:
        sl = slice(b, b + n)
        tx_n, ty_n = (W + tile - 1) // tile, (H + tile - 1) // tile
        f, _ = O.footprints(X[:, sl], C[sl].reshape(1, -1), R[sl], (nc, H, W), max_pixel_radius)
        pxc, pyc, rx, ry, ell = (f[:, k].astype(np.int64) for k in range(5))
        x0 = np.maximum(pxc - rx, 0)
        x1 = np.minimum(pxc + rx, W - 1)
        y0 = np.maximum(pyc - ry, 0)
        y1 = np.minimum(pyc + ry, H - 1)
        ch = C[sl].astype(np.int64)
        valid = (ch >= 0) & (ch < nc) & (rx >= 0) & (ry >= 0) & (x0 <= x1) & (y0 <= y1)
        wide = valid & ((rx > apron) | (ry > apron))
        pcx = np.clip(pxc, 0, W - 1)
        pcy = np.clip(pyc, 0, H - 1)
        t = tile_base + (np.where(valid, ch, 0) * ty_n + pcy // tile) * tx_n + pcx // tile
        dy0 = _corner_offset(pyc, H, X[1, sl])
        cls = row_class(M[0, 0, sl], M[0, 1, sl], M[1, 0, sl], M[1, 1, sl], dy0, W, H, rx,
                        x0 - pxc, x1 - pxc, y0 - pyc, y1 - pyc)
        cls = np.where(ell != 0, cls, 63) if class_bits == 6 else np.zeros_like(cls)
        k = (t << class_bits) | cls
        keys[sl] = np.where(~valid, key_invalid, np.where(wide, key_big, k))
        b += n
        tile_base += nc * ty_n * tx_n
    return keys, n_tiles
