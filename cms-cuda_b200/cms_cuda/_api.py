"""
Public entry points, with the reference's signatures and return types
(cms-cuda/_api.py:41-133).

``device`` accepts "auto", "cuda" and "gpu" (optionally "cuda:N"); every
value runs the CUDA library -- there is no CPU path, so "cpu" is rejected
with ValueError and a missing GPU raises RuntimeError.
"""

import functools

from . import _lib
from .calculator import MolecularSurfaceCalculator


@functools.lru_cache(maxsize=1)
def gpu_available():
    """True when the CUDA library loads and at least one CUDA device is visible."""
    return _lib.device_count() > 0


def _device_index(device):
    d = "auto" if device is None else str(device).lower()
    if d in ("auto", "cuda", "gpu"):
        idx = 0
    elif d.startswith("cuda:"):
        idx = int(d.split(":", 1)[1])
    elif d == "cpu":
        raise ValueError("device='cpu' is not supported: this implementation has no CPU path; "
                         "use device='auto', 'cuda' or 'gpu'")
    else:
        raise ValueError("device must be 'auto', 'cuda' or 'gpu', got %r" % (device,))
    if not gpu_available():
        raise RuntimeError("no CUDA GPU is usable (device=%r): the CUDA library needs a visible NVIDIA GPU" % (device,))
    return idx


def calculate_contact_ms(binder_xyz, binder_radii, target_xyz, target_radii, device="auto"):
    """
    Contact molecular surface of the binder against the target.

    Returns (cms: float, per_atom_target_cms: ndarray (N_target,), calc).
    Use calc.calc_contact_molecular_surface(target_side=False) for the binder side.
    """
    calc = MolecularSurfaceCalculator(_device_index(device))
    calc.add_binder_and_target(binder_xyz, binder_radii, target_xyz, target_radii)
    cms, per_atom_target_cms = calc.CalcLoaded()
    return cms, per_atom_target_cms, calc


def calculate_shape_complementarity(binder_xyz, binder_radii, target_xyz, target_radii, device="auto"):
    """
    Lawrence & Colman shape complementarity.

    Returns (sc, sc_int_area, median_dist, calc).
    """
    calc = MolecularSurfaceCalculator(_device_index(device))
    calc.add_binder_and_target(binder_xyz, binder_radii, target_xyz, target_radii)
    sc, sc_int_area, median_dist = calc.CalcLoadedSC()
    return sc, sc_int_area, median_dist, calc


def calculate_maximum_possible_contact_ms(xyz, radii, device="auto"):
    """
    Maximum possible CMS of one molecule (its distance-unweighted surface area).

    Returns (cms: float, per_atom: ndarray (N,), calc).
    """
    calc = MolecularSurfaceCalculator(_device_index(device))
    calc.AddMolecule(0, xyz, radii)
    cms, per_atom = calc.CalcLoadedMaxPossibleCMS()
    return cms, per_atom, calc
