"""openaccel_b200: B200-native (sm_100a) CVFEM assembly and SIMPLE
pressure-correction engine behind OpenAccel's assembler / linear-system API.

The compute path is the CUDA library built from ``openaccel_b200/csrc`` and
reached through the C-ABI of ``include/openaccel_b200.h`` (see ``runtime``).
"""
from . import meshgen  # noqa: F401
from .runtime import (  # noqa: F401
    OA_PREC_FP64,
    OA_PREC_MIXED,
    Flow,
    FlowSettings,
    Mesh,
    OpenAccelError,
    default_settings,
    lib,
)

__version__ = "0.1.0"
