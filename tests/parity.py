"""
Comparison helpers shared by the parity tests.

Integer / flag / index arrays must match exactly; floating-point arrays must
agree to TOL relative, scaled as max(1, |a|, |b|) so that tiny values are
compared absolutely (the convention of the reference's parity test,
test/test_gpu_parity.py:127-139, tightened from 1e-9 to 1e-12).
"""

import os

import numpy as np

TOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

FULL_CASES = ("golden_pkl", "synth_small_s7", "synth_zero_radii")
ALL_CASES = FULL_CASES + ("sc_example_pdb", "smallmol_7jkv_pdb", "synth_plain_1200_450", "synth_plain_8000_1800")


def load_case(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def inputs(case):
    return case["bx"], case["br"], case["tx"], case["tr"]


def exact(label, a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{label}: shape {a.shape} != {b.shape}"
    if a.dtype.kind == "f" or b.dtype.kind == "f":
        ok = np.array_equal(a, b, equal_nan=True)
    else:
        ok = np.array_equal(a, b)
    if not ok:
        if a.shape:
            bad = np.argwhere(np.asarray(a != b).reshape(a.shape))
            raise AssertionError(f"{label}: values differ at {len(bad)} positions, first {bad[:5].tolist()}")
        raise AssertionError(f"{label}: {a!r} != {b!r}")


def close(label, a, b, tol=TOL):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, f"{label}: shape {a.shape} != {b.shape}"
    if a.size == 0:
        return 0.0
    assert np.array_equal(np.isnan(a), np.isnan(b)), f"{label}: NaN layout differs"
    d = np.abs(np.nan_to_num(a) - np.nan_to_num(b))
    scale = np.maximum(1.0, np.maximum(np.abs(np.nan_to_num(a)), np.abs(np.nan_to_num(b))))
    worst = float((d / scale).max())
    assert worst <= tol, f"{label}: max scaled difference {worst:.3g} > {tol:g}"
    return worst
