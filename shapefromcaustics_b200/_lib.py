"""ctypes binding of ``libpds_b200.so`` (the C ABI declared in ``include/pds_b200.h``).

The library is the only compute path: if it is missing or fails to load, every op raises.
There is no CPU or eager-PyTorch fallback.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpds_b200.so")

PDS_OK = 0
PDS_ERR_INVALID_ARGUMENT = 1
PDS_ERR_WORKSPACE = 2
PDS_ERR_CUDA = 3
PDS_ERR_UNSUPPORTED = 4


class PdsConfig(ctypes.Structure):
    """Mirror of ``pds_config``."""
    _fields_ = [("tile", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("class_bits", ctypes.c_int32), ("apron_max", ctypes.c_int32),
                ("walk", ctypes.c_int32), ("min_blocks", ctypes.c_int32),
                ("coop_radius", ctypes.c_int32)]


class PdsSim(ctypes.Structure):
    """Mirror of ``pds_sim`` (56 bytes)."""
    _fields_ = [("photon_begin", ctypes.c_int64), ("n_photons", ctypes.c_int64),
                ("image_offset", ctypes.c_int64), ("channels", ctypes.c_int32),
                ("height", ctypes.c_int32), ("width", ctypes.c_int32),
                ("tiles_x", ctypes.c_int32), ("tiles_y", ctypes.c_int32),
                ("tile_base", ctypes.c_int32), ("reserved", ctypes.c_int32 * 2)]


assert ctypes.sizeof(PdsSim) == 56


class PdsPlate(ctypes.Structure):
    """Mirror of ``pds_plate``."""
    _fields_ = [("texel", ctypes.c_float), ("ior", ctypes.c_float),
                ("receiver_distance", ctypes.c_float), ("receiver_half", ctypes.c_float),
                ("light_dir", ctypes.c_float * 3), ("du0", ctypes.c_float)]

class PdsPointLight(ctypes.Structure):
    """Mirror of ``pds_point_light``."""
    _fields_ = [("position", ctypes.c_float * 3), ("plane_z", ctypes.c_float),
                ("xmin", ctypes.c_float), ("ymin", ctypes.c_float), ("xmax", ctypes.c_float),
                ("ymax", ctypes.c_float), ("smoothing", ctypes.c_float),
                ("energy", ctypes.c_float), ("simulations", ctypes.c_int32),
                ("inner", ctypes.c_int32), ("wavelengths", ctypes.c_int32)]


class PdsLandweber(ctypes.Structure):
    """Mirror of ``pds_landweber``."""
    _fields_ = [("tau", ctypes.c_float), ("shrink", ctypes.c_float), ("lower", ctypes.c_float),
                ("upper", ctypes.c_float), ("d1", ctypes.c_float), ("d2", ctypes.c_float),
                ("gamma", ctypes.c_float), ("radius", ctypes.c_int32)]


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t
_CFG = ctypes.POINTER(PdsConfig)

# name -> (restype, argtypes)
SIGNATURES = {
    "pds_last_error": (ctypes.c_char_p, []),
    "pds_version": (ctypes.c_char_p, []),
    "pds_workspace_bytes": (_SZ, [_I64, _I64, _I64, _I64, _CFG]),
    "pds_forward_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _I32, _P, _P,
                                       _SZ, _CFG, _P]),
    "pds_backward_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _I32, _P,
                                        _P, _P, _P, _SZ, _CFG, _P]),
    "pds_plan_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _I32, _P, _SZ,
                                    _CFG, _P]),
    "pds_forward_planned_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _I32,
                                               _P, _P, _SZ, _CFG, _P]),
    "pds_backward_planned_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I64, _I64,
                                                _I32, _P, _P, _P, _P, _SZ, _CFG, _P]),
    "pds_batch_layout": (ctypes.c_int, [ctypes.POINTER(PdsSim), _I32, _CFG,
                                        ctypes.POINTER(_I64)]),
    "pds_batch_image_elems": (ctypes.c_int, [ctypes.POINTER(PdsSim), _I32,
                                             ctypes.POINTER(_I64)]),
    "pds_batch_workspace_bytes": (_SZ, [_I64, _I64, _CFG]),
    "pds_batch_plan_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _P, _I32, _I64, _I32, _P, _SZ,
                                          _CFG, _P]),
    "pds_batch_forward_planned_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _P, _I32, _I64,
                                                     _I64, _I32, _P, _P, _SZ, _CFG, _P]),
    "pds_batch_backward_planned_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I64, _P, _I32,
                                                      _I64, _I64, _I32, _P, _P, _P, _P, _SZ, _CFG,
                                                      _P]),
    "pds_refract_forward_f32": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(PdsPlate), _P, _P,
                                               _P, _P, _I64, _P, _P, _P, _P, _P, _P]),
    "pds_refract_backward_f32": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(PdsPlate), _P, _P,
                                                _P, _I64, _P, _P, _P, _P, _P]),
    "pds_batch_refract_forward_f32": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P, _P, _P,
                                                     _P, _I64, _P, _P, _P, _P, _P, _P]),
    "pds_batch_refract_backward_f32": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P, _P, _P,
                                                      _I64, _P, _P, _P, _P, _P]),
    "pds_refract_backward_planned_f32": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(PdsPlate),
                                                        _P, _P, _P, _I64, _I64, _I64, _I64, _P,
                                                        _SZ, _CFG, _P, _P]),
    "pds_batch_refract_backward_planned_f32": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P,
                                                              _P, _P, _I64, _I64, _P, _SZ, _CFG,
                                                              _P, _P]),
    "pds_refract_point_forward_f32": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(PdsPlate),
                                                     ctypes.POINTER(PdsPointLight), _P, _P, _P,
                                                     _P, _P, _I64, _P, _P, _P, _P, _P, _P]),
    "pds_refract_point_backward_f32": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(PdsPlate),
                                                      ctypes.POINTER(PdsPointLight), _P, _P, _P,
                                                      _P, _I64, _P, _P, _P, _P, _P]),
    "pds_photon_source_f32": (ctypes.c_int, [_I32, _I32, _I32, ctypes.c_float, ctypes.c_uint64,
                                             ctypes.c_uint64, _P, _P, _P]),
    "pds_point_light_source_f32": (ctypes.c_int, [ctypes.POINTER(PdsPointLight), _I64,
                                                   ctypes.c_uint64, ctypes.c_uint64, _P, _P, _P,
                                                   _P, _P, _P]),
    "pds_landweber_workspace_bytes": (_SZ, [_I64, _I64]),
    "pds_landweber_update_f32": (ctypes.c_int, [_P, _P, _P, _I64, _I64,
                                                ctypes.POINTER(PdsLandweber), _P, _SZ, _P]),
    "pds_landweber_update_noalloc_f32": (ctypes.c_int, [_P, _P, _P, _I64, _I64,
                                                        ctypes.POINTER(PdsLandweber), _P]),
    "pds_plan_export": (ctypes.c_int, [_P, _SZ, _I64, _I64, _I32, _CFG, _P, _P, _P]),
}

_lib = None
_lock = threading.Lock()


class PdsError(RuntimeError):
    """A failure reported by the library (carries the PDS_ERR_* code)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library; raises ImportError if it has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.isfile(LIB_PATH):
                    raise ImportError(
                        f"{LIB_PATH} is missing: build it with "
                        "`python -m shapefromcaustics_b200.build` (nvcc, sm_100a)")
                l = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(l, name)
                    f.restype = res
                    f.argtypes = args
                _lib = l
    return _lib


def check(rc):
    if rc != PDS_OK:
        msg = lib().pds_last_error().decode(errors="replace")
        raise PdsError(rc, msg)


def config(tile=0, chunk=0, class_bits=0, apron_max=0, walk=0, min_blocks=0, coop_radius=0):
    return PdsConfig(int(tile), int(chunk), int(class_bits), int(apron_max), int(walk),
                     int(min_blocks), int(coop_radius))
