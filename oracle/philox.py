"""Philox4x32-10 and the plate's jittered photon entry points, in numpy. TEST INFRASTRUCTURE
ONLY: the checker of the device photon source (``pds_photon_source_f32``).

Philox4x32 with 10 rounds is restated from its publication (Salmon, Moraes, Dror, Shaw:
"Parallel random numbers: as easy as 1, 2, 3", SC 2011): per round the counter words
(c0, c1, c2, c3) become (hi(M1 c2) ^ c1 ^ k0, lo(M1 c2), hi(M0 c0) ^ c3 ^ k1, lo(M0 c0)) and the
key is bumped by the Weyl constants (W0, W1). The entry points follow the reference's
per-pixel random surface samples (``model/caustics.py:78-83``): one uniform offset in
[-1/2, 1/2) texel per axis.
"""
import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """ctr: (4, n) uint64 array of 32-bit words, key: (k0, k1) ints -> (4, n) uint64."""
    c = [np.asarray(w, dtype=np.uint64) & MASK for w in ctr]
    k0, k1 = np.uint64(key[0] & MASK), np.uint64(key[1] & MASK)
    for _ in range(10):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(MASK)
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & np.uint64(MASK)
        k1 = (k1 + np.uint64(W1)) & np.uint64(MASK)
    return np.stack(c)


def photon_source(rows, cols, per_texel, texel, seed, offset):
    """(px, py) float32 [rows * cols * per_texel]: photons 2j, 2j + 1 from counter block
    offset + j (words 0, 1 and 2, 3), offsets from the top 24 bits of each word; photon i in
    texel i % (rows * cols) (per_texel samples of one photon per texel, raster order)."""
    n = rows * cols * per_texel
    pairs = (n + 1) // 2
    ctr = np.uint64(offset) + np.arange(pairs, dtype=np.uint64)
    zero = np.zeros(pairs, dtype=np.uint64)
    r = philox4x32_10([ctr & np.uint64(MASK), ctr >> np.uint64(32), zero, zero],
                      (seed & MASK, (seed >> 32) & MASK))
    u = np.empty((2, 2 * pairs), dtype=np.uint64)
    u[0, 0::2], u[1, 0::2], u[0, 1::2], u[1, 1::2] = r[0], r[1], r[2], r[3]
    j = (u[:, :n] >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    j = j - np.float32(0.5)
    t = np.arange(n) % (rows * cols)
    iy = (t // cols).astype(np.float32)
    ix = (t % cols).astype(np.float32)
    cx, cy = np.float32(0.5 * (cols - 1)), np.float32(0.5 * (rows - 1))
    px = ((ix + j[0]) - cx) * np.float32(texel)
    py = ((iy + j[1]) - cy) * np.float32(texel)
    return px.astype(np.float32), py.astype(np.float32)
