"""
cms_cuda -- contact molecular surface (CMS) and Lawrence & Colman shape
complementarity (SC) on NVIDIA B200 (sm_100a).

Drop-in for the public API of ullahsamee/cms-cuda (cms-cuda/__init__.py):
``calculate_contact_ms``, ``calculate_shape_complementarity``,
``calculate_maximum_possible_contact_ms``, ``get_radii_from_names``,
``MolecularSurfaceCalculator`` (alias ``MolecularSurfaceCalculatorGPU``) and
``gpu_available``.  Everything runs in hand-written CUDA kernels behind the C
ABI of ``libcms_b200.so``; batched evaluation of many complexes is in
``cms_cuda.batch``.
"""

__version__ = "0.1.0"

from .radii import get_radii_from_names
from .calculator import MolecularSurfaceCalculator, MolecularSurfaceCalculatorGPU
from ._api import (
    calculate_contact_ms,
    calculate_shape_complementarity,
    calculate_maximum_possible_contact_ms,
    gpu_available,
)

__all__ = [
    "calculate_contact_ms",
    "calculate_shape_complementarity",
    "get_radii_from_names",
    "calculate_maximum_possible_contact_ms",
    "MolecularSurfaceCalculator",
    "MolecularSurfaceCalculatorGPU",
    "gpu_available",
]
