"""Python face of the CPU oracle (``oracle/pds_oracle.c``). TEST INFRASTRUCTURE ONLY.

Only the test suite, the smoke check and the benchmark's CPU-baseline leg use this module;
the product never imports it. The C restatement follows the reference's
``PyOptix/kernel/photon_differentials.cu`` (forward :60-113, backward :136-221); see the
header of ``pds_oracle.c`` for the two arithmetic modes.

Arrays use the reference's layouts: ``Ep[N]``, ``xp[2,N]``, ``Mp[2,3,N]``, ``cp[1,N]``
(int64), ``radius[N]``, images ``[C,H,W]``. Real inputs are taken as float64 (float32 values
convert exactly), so finite-difference checks may perturb below float32 resolution.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libpds_oracle.so")
SRC = os.path.join(HERE, "pds_oracle.c")

FP64 = 0
REF32 = 1
_MODES = {"fp64": FP64, "ref32": REF32}

_lib = None


def build(force=False):
    """Compile the oracle with gcc (OpenMP, no FMA contraction, no fast-math)."""
    if not force and os.path.isfile(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-o", LIB, SRC, "-lm"]
    subprocess.check_call(cmd)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        l = ctypes.CDLL(LIB)
        p, i64, i32, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int
        l.pds_oracle_forward.argtypes = [p, p, p, p, p, i64, i64, i64, i64, i32, i, i, p]
        l.pds_oracle_forward.restype = None
        l.pds_oracle_backward.argtypes = [p, p, p, p, p, p, i64, i64, i64, i64, i32, i, i, p, p, p]
        l.pds_oracle_backward.restype = None
        l.pds_oracle_footprints.argtypes = [p, p, p, i64, i64, i64, i64, i32, p, p]
        l.pds_oracle_footprints.restype = None
        _lib = l
    return _lib


def _f64(a):
    """float64 copy; float32 inputs convert exactly, so footprints match the reference's."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _inputs(Ep, xp, Mp, cp, radius):
    E = _f64(Ep).reshape(-1)
    N = E.shape[0]
    X = _f64(xp).reshape(2, N)
    M = _f64(Mp).reshape(2, 3, N)
    C = np.ascontiguousarray(np.asarray(cp, dtype=np.int64)).reshape(1, N)
    R = _f64(radius).reshape(N)
    return E, X, M, C, R, N


def forward(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius, mode="fp64", threads=0):
    """Oracle of ``pds_forward`` -> float64 image ``[C,H,W]``."""
    E, X, M, C, R, N = _inputs(Ep, xp, Mp, cp, radius)
    nc, h, w = (int(v) for v in output_size)
    out = np.empty((nc, h, w), dtype=np.float64)
    lib().pds_oracle_forward(_ptr(E), _ptr(X), _ptr(M), _ptr(C), _ptr(R), N, nc, h, w,
                             int(max_pixel_radius), _MODES[mode], int(threads), _ptr(out))
    return out


def backward(grad, Ep, xp, Mp, cp, radius, max_pixel_radius, mode="fp64", threads=0):
    """Oracle of ``pds_backward`` -> float64 ``(grad_Ep[N], grad_xp[2,N], grad_Mp[2,3,N])``."""
    E, X, M, C, R, N = _inputs(Ep, xp, Mp, cp, radius)
    G = np.ascontiguousarray(np.asarray(grad, dtype=np.float64))
    nc, h, w = G.shape
    gE = np.empty(N, dtype=np.float64)
    gX = np.empty((2, N), dtype=np.float64)
    gM = np.empty((2, 3, N), dtype=np.float64)
    lib().pds_oracle_backward(_ptr(G), _ptr(E), _ptr(X), _ptr(M), _ptr(C), _ptr(R), N, nc, h,
                              w, int(max_pixel_radius), _MODES[mode], int(threads), _ptr(gE),
                              _ptr(gX), _ptr(gM))
    return gE, gX, gM


def footprints(xp, cp, radius, output_size, max_pixel_radius):
    """Per photon ``(px_c, py_c, rx, ry, ellipse_all)`` and in-image box pixel counts."""
    X = _f64(xp)
    N = X.shape[-1]
    X = X.reshape(2, N)
    C = np.ascontiguousarray(np.asarray(cp, dtype=np.int64)).reshape(N)
    R = _f64(radius).reshape(N)
    nc, h, w = (int(v) for v in output_size)
    out5 = np.empty((N, 5), dtype=np.int32)
    box = np.empty(N, dtype=np.int64)
    lib().pds_oracle_footprints(_ptr(X), _ptr(C), _ptr(R), N, nc, h, w, int(max_pixel_radius),
                                _ptr(out5), _ptr(box))
    return out5, box
