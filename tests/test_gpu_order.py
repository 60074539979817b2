"""
AddMolecule in any order (reference cms-cuda/_core.py:923-943 accepts the
target before the binder, and split calls).

The fixture synth_small_s7_order.npz holds the reference's own run with the
molecules of synth_small_s7 added target first, and interleaved
(binder part, target part, binder rest, target rest).  Its surfaces, SC and
run state (natom numbering in call order) must match exactly / within 1e-12.

The reference's target-side readout indexes per-atom bins by natom minus the
molecule-0 count (_core.py:990-995), so with target atoms numbered before
binder atoms its np.bincount raises ValueError (recorded in the fixture).
Here both per-atom readouts list one molecule's atoms in the order they were
added; the target side is checked against the binder-first reference run
(the surfaces are identical, only the numbering differs), and the binder
side against the reference's own N-long bincount at the binder positions.
"""

import numpy as np
import pytest

from parity import close, exact, inputs, load_case

pytestmark = pytest.mark.gpu

ORDER_CASES = {
    "target_first": ((1, "t", 0, None), (0, "b", 0, None)),
    "interleaved": ((0, "b", 0, 70), (1, "t", 0, 150), (0, "b", 70, None), (1, "t", 150, None)),
}


@pytest.fixture(scope="module")
def cases():
    return load_case("synth_small_s7"), load_case("synth_small_s7_order")


@pytest.mark.parametrize("name", sorted(ORDER_CASES))
def test_out_of_order_molecules(cases, name):
    from cms_cuda import MolecularSurfaceCalculator
    base, ref = cases
    bx, br, tx, tr = inputs(base)
    src = {"b": (bx, br), "t": (tx, tr)}
    calc = MolecularSurfaceCalculator()
    mol_of_call = []
    for mol, side, a, b in ORDER_CASES[name]:
        x, r = src[side]
        calc.AddMolecule(mol, x[a:b], r[a:b])
        mol_of_call += [mol] * len(r[a:b])
    mol_of_call = np.array(mol_of_call)
    assert ref[f"{name}_target_raises"]

    cms, pa = calc.CalcLoaded()
    close("target cms (binder-first reference)", cms, base["cms"])
    close("target per-atom (binder-first reference)", pa, base["per_atom_target"])
    bcms, pb = calc.calc_contact_molecular_surface(target_side=False)
    close("binder cms", bcms, ref[f"{name}_cms_binder"])
    binder_pos = np.nonzero(mol_of_call == 0)[0]
    close("binder per-atom", pb, ref[f"{name}_per_atom_binder"][binder_pos])
    sc = calc.CalcLoadedSC()
    close("sc", np.array(sc), ref[f"{name}_sc"])

    r = calc.run
    exact("molecule", r.atoms.molecule, ref[f"{name}_molecule"])
    exact("atten", r.atoms.atten, ref[f"{name}_atten"])
    exact("access", r.atoms.access, ref[f"{name}_access"])
    for m in (0, 1):
        d = r.dots[m]
        exact(f"dots[{m}].atom_idx", d.atom_idx, ref[f"{name}_dots{m}_atom"])
        exact(f"dots[{m}].buried", d.buried, ref[f"{name}_dots{m}_buried"])
        close(f"dots[{m}].coor_xyz", d.coor_xyz, base[f"dots{m}_coor"])
        close(f"dots[{m}].area", d.area, base[f"dots{m}_area"])
        exact(f"trimmed[{m}].atom_idx", r.trimmed_dots[m].atom_idx, ref[f"{name}_trim{m}_atom"])
    p = r.probes
    exact("probe atoms", np.stack([p.atom_idx_0, p.atom_idx_1, p.atom_idx_2], 1), ref[f"{name}_probe_atoms"])
    close("probe points", p.point_xyz, ref[f"{name}_probe_point"])
    tq = r.toroid_queue
    exact("toroid atoms", np.array([(t[0], t[1]) for t in tq], dtype=np.int32).reshape(-1, 2),
          ref[f"{name}_tor_atoms"])
    close("toroid centres", np.array([t[3] for t in tq]).reshape(-1, 3), ref[f"{name}_tor_tij"])
    exact("neighbour rows", r.neighbor_array.natom, ref[f"{name}_nb_natom"])
    exact("neighbour counts", r.neighbor_array.nneighbors, ref[f"{name}_nb_count"])
    exact("buried rows", r.buried_array.natom, ref[f"{name}_bu_natom"])

    # the gradient comes back in AddMolecule order: rows equal the binder-first run's rows, moved
    plain = MolecularSurfaceCalculator()
    plain.add_binder_and_target(bx, br, tx, tr)
    plain.CalcLoaded()
    g0 = plain.calc_contact_molecular_surface_gradient(True)
    g = calc.calc_contact_molecular_surface_gradient(True)
    order = np.concatenate([np.nonzero(mol_of_call == 0)[0], np.nonzero(mol_of_call == 1)[0]])
    exact("gradient rows", g[order], g0)
