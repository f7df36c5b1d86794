"""The allocation-free Landweber update (pds_landweber_update_noalloc_f32), called through the
C ABI, against the workspace entry point (pds_landweber_update_f32) on the same inputs.

That entry point exists for callers that cannot allocate device memory (their device memory
belongs to another allocator, or their loop may not allocate after start-up); its scratch is
a static device array of the library, so it takes no workspace. This file is collected last
so that a run stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

from shapefromcaustics_b200 import _lib
from shapefromcaustics_b200.landweber import LandweberParams

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, as the other Landweber update tests


def _field(rows, cols, seed):
    g = torch.Generator().manual_seed(seed)
    d = torch.rand((rows, cols), generator=g) * 0.2
    grad = torch.randn((rows, cols), generator=g)
    mask = (torch.rand((rows, cols), generator=g) > 0.3).float()
    s = float((mask * d).sum())
    p = LandweberParams(tau=0.05, alpha=0.1, lower=0.0, upper=0.15, d1=2 * s, d2=3 * s,
                        gamma=0.1, radius=2).c_struct()
    return d.cuda(), grad.cuda(), mask.cuda(), p


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _with_workspace(d, grad, mask, p, stream):
    lib = _lib.lib()
    rows, cols = d.shape
    ws = torch.empty(int(lib.pds_landweber_workspace_bytes(rows, cols)), dtype=torch.uint8,
                     device="cuda")
    out = d.clone()
    _lib.check(lib.pds_landweber_update_f32(_p(out), _p(grad), _p(mask), rows, cols,
                                            ctypes.byref(p), _p(ws), ws.numel(), stream))
    return out


def _no_alloc(d, grad, mask, p, stream):
    lib = _lib.lib()
    rows, cols = d.shape
    out = d.clone()
    _lib.check(lib.pds_landweber_update_noalloc_f32(_p(out), _p(grad), _p(mask), rows, cols,
                                                    ctypes.byref(p), stream))
    return out


def rel_l2(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_no_alloc_update_matches_workspace_update_twice(cuda):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row, the second on a smaller field: it must not see the first call's
    # scratch contents
    for rows, cols, seed in ((700, 1100, 1), (257, 131, 2)):
        d, grad, mask, p = _field(rows, cols, seed)
        ref = _with_workspace(d, grad, mask, p, stream)
        got = _no_alloc(d, grad, mask, p, stream)
        torch.cuda.synchronize()
        assert rel_l2(got, ref) <= TOL


def test_no_alloc_rejects_fields_beyond_its_scratch(cuda):
    lib = _lib.lib()
    p = LandweberParams(d1=1.0, d2=2.0).c_struct()
    x = torch.zeros(1, device="cuda")
    rc = lib.pds_landweber_update_noalloc_f32(_p(x), _p(x), _p(x), 1025, 1024, ctypes.byref(p),
                                              None)
    assert rc == _lib.PDS_ERR_UNSUPPORTED
    assert b"exceeds its static scratch" in lib.pds_last_error()
