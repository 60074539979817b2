"""
Host-side logic that runs without a GPU: the C-ABI library loads and exports
every symbol include/cms_b200.h declares, the radii table / wildcard matcher,
the PDB reader, the synthetic generator and the API's device handling.
"""

import ctypes
import os
import re

import numpy as np
import pytest

from parity import load_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "cms_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cms_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from cms_cuda import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) == set(_lib.EXPORTED)


def test_library_loads_without_gpu():
    from cms_cuda import _lib
    lib = _lib.load()
    assert lib.cms_version().decode().startswith("cms_b200")
    assert _lib.device_count() >= 0


def test_radii_known_values():
    from cms_cuda import get_radii_from_names
    r = get_radii_from_names(["ALA", "ARG", "ARG", "GLY", "LIG", "LIG", "LIG", "XYZ", "HOH", "LGA", "TRP"],
                             ["CB", "NH1", "CZ", "CA", "C1", "N7", "O2", "P", "O", "AROC", "CZ2"])
    np.testing.assert_array_equal(r, [1.95, 1.70, 1.80, 1.90, 1.85, 1.65, 1.60, 2.15, 1.70, 2.00, 1.90])
    # unmatched names get 0, hydrogens 0.5
    r = get_radii_from_names(["ALA", "ALA", "ALA"], ["ZZ", "H", "1HB"])
    np.testing.assert_array_equal(r, [0.0, 0.5, 0.5])


def test_wildcard_match_semantics():
    from cms_cuda.radii import wildcard_match
    assert wildcard_match("P", "P*", 3)          # trailing * matches an exhausted query
    assert not wildcard_match("PB", "P", 4)
    assert wildcard_match("NH2", "NH*", 5)
    assert not wildcard_match("N", "NH*", 3)


def test_radii_of_golden_inputs():
    """PDB-derived radii of the golden fixtures equal the reference's."""
    from cms_cuda.structure import read_pdb_chains
    from cms_cuda import get_radii_from_names
    case = load_case("sc_example_pdb")
    ref = os.environ.get("CMS_REFERENCE_DIR")
    pdb = os.path.join(ref, "test", "sc_example.pdb") if ref else ""
    if not os.path.exists(pdb):
        pytest.skip("no reference checkout named by CMS_REFERENCE_DIR")
    ch = read_pdb_chains(pdb)
    np.testing.assert_array_equal(get_radii_from_names(ch["B"][1], ch["B"][2]), case["br"])
    np.testing.assert_array_equal(ch["A"][0], case["tx"])


def test_synthetic_generator_is_seeded_and_well_formed():
    from cms_cuda import synth
    b1 = synth.make_batch([300, 500], [100, 40], seed=5, ligand=[False, True])
    b2 = synth.make_batch([300, 500], [100, 40], seed=5, ligand=[False, True])
    np.testing.assert_array_equal(b1.xyz, b2.xyz)
    np.testing.assert_array_equal(b1.radius, b2.radius)
    assert b1.N == 940 and list(b1.atom_off) == [0, 400, 940]
    for c in range(2):
        bx, br, tx, tr = b1.complex(c)
        d = np.sqrt(((bx[:, None] - tx[None]) ** 2).sum(-1)).min()
        assert 3.5 - 1e-6 <= d <= 4.5 + 1e-6
        assert (br > 0).all() and (tr > 0).all()
    # ligand binder atoms carry HETATM C*/N*/O* radii
    assert set(np.round(b1.complex(1)[1], 2)) <= {1.85, 1.65, 1.60}


def test_api_rejects_cpu_device():
    from cms_cuda import calculate_contact_ms
    with pytest.raises(ValueError):
        calculate_contact_ms(np.zeros((1, 3)), np.ones(1), np.ones((1, 3)), np.ones(1), device="cpu")
    with pytest.raises(ValueError):
        calculate_contact_ms(np.zeros((1, 3)), np.ones(1), np.ones((1, 3)), np.ones(1), device="tpu")


def test_gpu_missing_raises_not_falls_back(monkeypatch):
    """Without a GPU the API raises instead of computing on the CPU."""
    import cms_cuda._api as api
    api.gpu_available.cache_clear()
    monkeypatch.setattr(api._lib, "device_count", lambda: 0)
    try:
        with pytest.raises(RuntimeError):
            api.calculate_contact_ms(np.zeros((1, 3)), np.ones(1), np.ones((1, 3)), np.ones(1))
    finally:
        api.gpu_available.cache_clear()


def test_stream_arguments_are_checked_before_any_gpu_work():
    """BatchCalculator.run_stream's argument check: one atom count, one float64 N x 3 buffer per batch."""
    from cms_cuda.batch import check_stream_args
    off = np.array([0, 3, 7]); nb = np.array([1, 2])
    b = (off, nb, np.zeros((7, 3)), np.ones(7))
    assert check_stream_args([b, b], [np.zeros((7, 3)), np.zeros((7, 3))]) == 7
    with pytest.raises(ValueError):
        check_stream_args([b, b], [np.zeros((7, 3))])
    with pytest.raises(ValueError):
        check_stream_args([b, (np.array([0, 3, 6]), nb, np.zeros((6, 3)), np.ones(6))], [np.zeros((7, 3))] * 2)
    with pytest.raises(ValueError):
        check_stream_args([b], [np.zeros((7, 3), np.float32)])
    with pytest.raises(ValueError):
        check_stream_args([b], [np.zeros((3, 7)).T])
    with pytest.raises(ValueError):
        check_stream_args([], [])
