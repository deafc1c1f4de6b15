"""B200-native lunarscout horizon-and-lighting hot path.

Hand-written sm_100a CUDA kernels (``csrc/``, built into ``libls200.so``)
behind a C ABI (``include/ls200.h``) and Python session classes that are
drop-ins for lunarscout's ``CudaSession``, ``LightmapCudaSession`` and
``PsrCudaSession``.  Importing this package does not initialise CUDA.
"""

from __future__ import annotations

from .contract import (
    AZIMUTH_COUNT,
    PATCH_SIZE,
    ContractConfiguration,
    DemGrid,
    HorizonBuffers,
    ProjectionParameters,
    PyramidArrays,
    SegmentTensor,
)

__all__ = [
    "AZIMUTH_COUNT",
    "PATCH_SIZE",
    "ContractConfiguration",
    "DemGrid",
    "HorizonBuffers",
    "ProjectionParameters",
    "PyramidArrays",
    "SegmentTensor",
]

__version__ = "0.1.0"
