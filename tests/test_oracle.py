"""
The CPU oracle (oracle/cms_oracle.py) pinned against the reference's outputs:
the golden fixtures (made from the reference calculator) and the reference's
own regression pickles (test/golden.pkl: cms 275.5999647907913; sc_golden.pkl:
sc 0.6297053428112819, area 529.8866053867879, distance 0.601465993751502).
The oracle must reproduce every array bit for bit.
"""

import numpy as np
import pytest

from oracle import cms_oracle as O
from parity import exact, inputs, load_case


@pytest.fixture(scope="module", params=["golden_pkl", "synth_small_s7"])
def oracle_run(request):
    case = load_case(request.param)
    out = O.run_complex(*inputs(case))
    mx, mpa, mS = O.run_max_cms(case["tx"], case["tr"])
    return case, out, (mx, mpa, mS)


def test_scalars(oracle_run):
    case, out, (mx, mpa, _) = oracle_run
    exact("cms", out["cms"], case["cms"])
    exact("cms binder", out["cms_binder"], case["cms_binder"])
    exact("sc", [out["sc"], out["sc_area"], out["sc_distance"]],
          [case["sc"], case["sc_area"], case["sc_distance"]])
    exact("per-atom", out["cms_per_atom"], case["per_atom_target"])
    exact("per-atom binder", out["cms_binder_per_atom"], case["per_atom_binder"])
    exact("max cms", mx, case["max_cms"])
    exact("max per-atom", mpa, case["per_atom_max"])


def test_large_complex():
    """The plain large complex (1800 + 8000 atoms) against the reference's own run of it."""
    case = load_case("synth_plain_8000_1800")
    out = O.run_complex(*inputs(case))
    exact("cms", out["cms"], case["cms"])
    exact("cms binder", out["cms_binder"], case["cms_binder"])
    exact("sc", [out["sc"], out["sc_area"], out["sc_distance"]],
          [case["sc"], case["sc_area"], case["sc_distance"]])
    exact("per-atom", out["cms_per_atom"], case["per_atom_target"])
    exact("per-atom binder", out["cms_binder_per_atom"], case["per_atom_binder"])
    S = out["surface"]
    exact("atten", S.atten, case["atten"])
    exact("access", S.access, case["access"])


def test_run_state(oracle_run):
    case, out, _ = oracle_run
    S = out["surface"]
    exact("atten", S.atten, case["atten"])
    exact("access", S.access, case["access"])
    exact("nn", S.nn, case["nn"])
    exact("nbur", S.nbur, case["nbur"])
    exact("neighbour rows", S.pad_id, case["nb_natom"])
    exact("buried rows", S.bpad_id, case["bu_natom"])
    exact("counts", [S.counts["convex"], S.counts["toroidal"], S.counts["concave"]], case["counts"])
    for m in (0, 1):
        d = S.dot_arrays[m]
        for k, f in (("coor", "coor"), ("nml", "nml"), ("area", "area"), ("buried", "buried"), ("type", "type"),
                     ("atom", "atom")):
            exact(f"dots{m}.{k}", d[f], case[f"dots{m}_{k}"])
    p = S.probes
    exact("probe atoms", np.stack([p["a0"], p["a1"], p["a2"]], 1), case["probe_atoms"])
    exact("probe point", p["point"], case["probe_point"])
    T = S.toroid
    exact("toroid", np.stack([T["i"], T["j"]], 1), case["tor_atoms"])
    exact("toroid tij", T["tij"], case["tor_tij"])
    surf = out["sc_details"]["surface"]
    for m in range(3):
        got = [surf[m][k] for k in ("d_mean", "d_median", "s_mean", "s_median", "trimmedArea", "nTrimmedDots",
                                    "nAllDots")]
        exact(f"surface[{m}]", got, case["surface"][m][:7])


def test_reference_pickles():
    case = load_case("golden_pkl")
    out = O.run_complex(*inputs(case))
    exact("golden.pkl cms", out["cms"], float(case["pkl_cms"]))
    exact("sc_golden.pkl", [out["sc"], out["sc_area"], out["sc_distance"]],
          [float(case["pkl_sc"]), float(case["pkl_sc_area"]), float(case["pkl_sc_distance"])])
    S = out["surface"]
    exact("golden.pkl dots", [len(S.dot_arrays[0]["area"]), len(S.dot_arrays[1]["area"])], case["pkl_dots"])
    exact("golden.pkl dot types", [S.counts["convex"], S.counts["toroidal"], S.counts["concave"]], case["pkl_counts"])
    tr = out["sc_details"]["trimmed"]
    exact("sc_golden.pkl trimmed", [len(tr[0]["area"]), len(tr[1]["area"])], case["pkl_trimmed"])


def test_binned_median_known_answers():
    # grouped-data median: bins of 0.02, linear interpolation inside the 50 % bin
    assert O.binned_median(np.array([]), 0.02) == 0.0
    v = np.array([0.01, 0.03, 0.05, 0.07])
    # bins 0,1,2,3 with 25 % each; 50 % reached at bin 1 -> 0.02 + (50-25)*0.02/25
    assert abs(O.binned_median(v, 0.02) - 0.04) < 1e-15


@pytest.mark.parametrize("slot", [0, 6])
def test_ligand_binders_of_the_batched_workload(slot):
    """Two ligand-binder complexes of the batched workload (HETATM C*/N*/O* radii) against the reference's run."""
    z = load_case("batched_4096_sample")
    assert bool(z["ligand"][slot])
    case = {k[len(f"k{slot}_"):]: v for k, v in z.items() if k.startswith(f"k{slot}_")}
    out = O.run_complex(*inputs(case))
    exact("cms", out["cms"], case["cms"])
    exact("cms binder", out["cms_binder"], case["cms_binder"])
    exact("sc", [out["sc"], out["sc_area"], out["sc_distance"]], [case["sc"], case["sc_area"], case["sc_distance"]])
    exact("per-atom", out["cms_per_atom"], case["per_atom_target"])
    S = out["surface"]
    for m in (0, 1):
        d = S.dot_arrays[m]
        exact(f"dots{m}.atom", d["atom"], case[f"dots{m}_atom"])
        exact(f"dots{m}.buried", d["buried"], case[f"dots{m}_buried"])
        exact(f"dots{m}.type", d["type"], case[f"dots{m}_type"])
