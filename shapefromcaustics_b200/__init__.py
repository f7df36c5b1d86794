"""B200-native (sm_100a) photon-differential splatting for ShapeFromCaustics.

Drop-in for the reference's ``PhotonDifferentialSplatting`` torch extension
(``pds_forward`` / ``pds_backward``) and its ``PDS`` autograd Function, backed by the C ABI
of ``libpds_b200.so`` (``include/pds_b200.h``).
"""
from .splatting import (BatchedSplat, SplatPlan, pds_backward, pds_forward,  # noqa: F401
                        set_default_config)
from .photon_differential import PDS, set_keep_plan  # noqa: F401
from . import shim  # noqa: F401

__version__ = "1.0.0"
