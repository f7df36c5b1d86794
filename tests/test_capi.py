"""The C ABI library loads without a GPU, exports every function include/pds_b200.h declares,
and rejects bad arguments before touching the device."""
import ctypes
import os
import re

import pytest

from shapefromcaustics_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(pds_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("pds_forward_f32", "pds_backward_f32", "pds_plan_f32", "pds_batch_layout",
              "pds_plan_export", "pds_last_error", "pds_workspace_bytes"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for n in declared_functions():
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_version_and_workspace_query():
    lib = _lib.lib()
    assert b"sm_100a" in lib.pds_version()
    a = lib.pds_workspace_bytes(1 << 20, 1, 512, 512, None)
    b = lib.pds_workspace_bytes(1 << 21, 1, 512, 512, None)
    assert 40 * (1 << 20) < a < b


def test_argument_errors_without_a_device():
    lib = _lib.lib()
    rc = lib.pds_forward_f32(None, None, None, None, None, 5, 1, 8, 8, 20, None, None, 0, None, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT
    assert b"null" in lib.pds_last_error()
    p = ctypes.c_void_p(16)
    cfg = _lib.config(tile=24)
    rc = lib.pds_plan_f32(p, p, p, p, p, 5, 1, 8, 8, 20, p, 1 << 20, ctypes.byref(cfg), None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"tile" in lib.pds_last_error()
    rc = lib.pds_plan_f32(p, p, p, p, p, 5, 0, 8, 8, 20, p, 1 << 20, None, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"positive" in lib.pds_last_error()
    rc = lib.pds_plan_f32(p, p, p, p, p, 5, 1, 8, 8, 20, p, 10, None, None)
    assert rc == _lib.PDS_ERR_WORKSPACE
    rc = lib.pds_plan_export(p, 10, 5, 1, 20, None, p, p, None)
    assert rc == _lib.PDS_ERR_WORKSPACE
    rc = lib.pds_plan_export(p, 1 << 20, 5, 1, 20, None, None, None, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"null" in lib.pds_last_error()


def test_batch_layout_on_host():
    lib = _lib.lib()
    t = (_lib.PdsSim * 3)()
    shapes = [(1, 512, 512), (2, 100, 70), (1, 16, 16)]
    b = off = 0
    for k, (c, h, w) in enumerate(shapes):
        t[k].photon_begin, t[k].n_photons = b, 10 + k
        t[k].channels, t[k].height, t[k].width = c, h, w
        t[k].image_offset = off
        b += 10 + k
        off += c * h * w
    nt = ctypes.c_int64()
    cfg = _lib.config(tile=32)
    _lib.check(lib.pds_batch_layout(t, 3, ctypes.byref(cfg), ctypes.byref(nt)))
    assert [t[k].tile_base for k in range(3)] == [0, 256, 256 + 2 * 4 * 3]
    assert nt.value == 256 + 24 + 1
    _lib.check(lib.pds_batch_layout(t, 3, None, ctypes.byref(nt)))  # default 64-pixel tiles
    assert [t[k].tile_base for k in range(3)] == [0, 64, 64 + 2 * 2 * 2]
    t[1].photon_begin = 3  # not contiguous
    with pytest.raises(_lib.PdsError):
        _lib.check(lib.pds_batch_layout(t, 3, None, ctypes.byref(nt)))


def test_batch_image_ranges_are_checked_on_host():
    lib = _lib.lib()
    t = (_lib.PdsSim * 3)()
    for k in range(3):
        t[k].photon_begin, t[k].n_photons = 5 * k, 5
        t[k].channels, t[k].height, t[k].width = 1, 32, 32
    # all three summed into one image
    n = ctypes.c_int64()
    _lib.check(lib.pds_batch_image_elems(t, 3, ctypes.byref(n)))
    assert n.value == 32 * 32
    # separate images with a gap
    t[1].image_offset, t[2].image_offset = 1024, 4096
    _lib.check(lib.pds_batch_image_elems(t, 3, ctypes.byref(n)))
    assert n.value == 4096 + 1024
    nt = ctypes.c_int64()
    _lib.check(lib.pds_batch_layout(t, 3, None, ctypes.byref(nt)))
    # a range that overlaps another without being the same image
    t[2].image_offset = 1500
    for call in (lambda: lib.pds_batch_image_elems(t, 3, ctypes.byref(n)),
                 lambda: lib.pds_batch_layout(t, 3, None, ctypes.byref(nt))):
        with pytest.raises(_lib.PdsError, match="overlap"):
            _lib.check(call())
    t[2].image_offset = -1
    with pytest.raises(_lib.PdsError, match="negative"):
        _lib.check(lib.pds_batch_image_elems(t, 3, ctypes.byref(n)))


def test_records_mode_argument_errors_without_a_device():
    # the refraction backward from a plan's gradient records: plate, gradient and workspace
    # are checked before anything is enqueued; a splat backward with some but not all of its
    # gradient outputs null is rejected (all null: the records mode)
    lib = _lib.lib()
    p = ctypes.c_void_p(256)
    plate = _lib.PdsPlate()
    plate.texel, plate.ior, plate.receiver_half, plate.receiver_distance = 0.1, 1.5, 10.0, 50.0
    rc = lib.pds_refract_backward_planned_f32(p, 8, 8, None, p, p, p, 5, 1, 8, 8, p, 1 << 20,
                                              None, p, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"plate" in lib.pds_last_error()
    rc = lib.pds_refract_backward_planned_f32(p, 8, 8, ctypes.byref(plate), p, p, p, 5, 1, 8, 8,
                                              p, 1 << 20, None, None, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"null" in lib.pds_last_error()
    rc = lib.pds_refract_backward_planned_f32(p, 8, 8, ctypes.byref(plate), p, p, p, 5, 1, 8, 8,
                                              p, 10, None, p, None)
    assert rc == _lib.PDS_ERR_WORKSPACE
    rc = lib.pds_refract_backward_planned_f32(p, 8, 8, ctypes.byref(plate), p, p, p, 5, 1, 8, 8,
                                              ctypes.c_void_p(16), 1 << 20, None, p, None)
    assert rc == _lib.PDS_ERR_WORKSPACE and b"aligned" in lib.pds_last_error()
    rc = lib.pds_batch_refract_backward_planned_f32(p, 8, 8, None, None, 0, p, p, p, 5, 4, p,
                                                    1 << 20, None, p, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"plate table" in lib.pds_last_error()
    rc = lib.pds_batch_refract_backward_planned_f32(p, 8, 8, p, p, 1, p, p, p, 5, 4, p, 10,
                                                    None, p, None)
    assert rc == _lib.PDS_ERR_WORKSPACE
    rc = lib.pds_backward_planned_f32(p, p, p, p, p, p, 5, 1, 8, 8, 20, p, None, None, p, 1 << 20,
                                      None, None)
    assert rc == _lib.PDS_ERR_INVALID_ARGUMENT and b"null gradient" in lib.pds_last_error()
