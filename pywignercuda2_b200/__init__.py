"""pywignercuda2_b200 -- B200-native (sm_100a) split-operator propagation of
4-D phase-space Wigner functions, a drop-in for the ``GPU_Wigner4D``,
``GPU_WignerDirac4D`` and ``GPU_WignerDiracKvN4D`` classes of
cabrer7/PyWignerCUDA2.

The numerical work runs in ``libwigner_b200.so`` (hand-written CUDA for
sm_100a behind a C ABI, ``include/wigner_b200.h``); this package holds the
reference-compatible Python classes that build its plans and call it.
"""
from ._lib import WignerError, load as load_library  # noqa: F401
from .device import DeviceScalar, GPUArray  # noqa: F401
from .wigner4d import GPU_Wigner4D  # noqa: F401
from .batch import WignerBatch  # noqa: F401

from .dirac4d import GPU_WignerDirac4D, GPU_WignerDiracKvN4D  # noqa: F401

__all__ = ["GPU_Wigner4D", "GPU_WignerDirac4D", "GPU_WignerDiracKvN4D", "WignerBatch", "GPUArray", "DeviceScalar",
           "WignerError", "load_library"]
