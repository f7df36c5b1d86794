"""Import shim: makes ``import PhotonDifferentialSplatting`` resolve to this library.

The reference's differentiable model imports its splatting ops with
``from PhotonDifferentialSplatting import pds_forward, pds_backward``
(``model/photon_differential.py:4``). After ``install()``, that import yields this library's
``pds_forward`` / ``pds_backward`` (same signatures and list returns), so the reference's
``PDS`` Function and Landweber loop run on the sm_100a kernels unmodified.
"""
import sys
import types

MODULE_NAME = "PhotonDifferentialSplatting"


def install():
    """Register the module alias (idempotent); returns the module object."""
    from . import splatting
    mod = sys.modules.get(MODULE_NAME)
    if mod is None or getattr(mod, "__pds_b200__", False) is False:
        mod = types.ModuleType(MODULE_NAME)
        mod.__doc__ = "pds_b200 stand-in for the reference's PhotonDifferentialSplatting module"
        mod.pds_forward = splatting.pds_forward
        mod.pds_backward = splatting.pds_backward
        mod.__pds_b200__ = True
        sys.modules[MODULE_NAME] = mod
    return mod
