"""
Heavy-atom loader (cms_cuda.loader) on hand-written PDB and mmCIF files with
the reference CLI's selection rules (examples/calculate_cms_sc.py:43-97):
first model only, one alternate location per atom (highest occupancy), water
and single-atom HETATM residues dropped unless kept, hydrogens dropped by
element or by name, chain / residue-name selection and exclusion.
"""

import numpy as np

PDB = """\
HEADER    TEST
MODEL        1
ATOM      1  N   ALA A   1       0.000   0.000   0.000  1.00  0.00           N
ATOM      2  CA  ALA A   1       1.458   0.000   0.000  1.00  0.00           C
ATOM      3  CB AALA A   1       1.988  -0.773   1.199  0.40  0.00           C
ATOM      4  CB BALA A   1       1.990  -0.770   1.210  0.60  0.00           C
ATOM      5  H   ALA A   1      -0.500   0.800   0.000  1.00  0.00           H
ATOM      6 1HB  ALA A   1       2.500  -0.200   1.900  1.00  0.00
ATOM      7  N   GLY A   1A      3.300   1.200  -0.500  1.00  0.00           N
ATOM      8  CA  GLY A   1A      4.700   1.300  -0.700  1.00  0.00           C
HETATM    9 ZN    ZN A 101       5.000   5.000   5.000  1.00  0.00          ZN
HETATM   10  O   HOH A 201       7.000   7.000   7.000  1.00  0.00           O
HETATM   11  C1  BTN A 301       8.000   1.000   2.000  1.00  0.00           C
HETATM   12  O1  BTN A 301       9.000   1.500   2.500  1.00  0.00           O
ATOM     13  N   SER B   5      10.000   0.000   0.000  1.00  0.00           N
ATOM     14  OG  SER B   5      11.000   0.500   0.000  1.00  0.00           O
ENDMDL
MODEL        2
ATOM     15  N   ALA A   1      50.000   0.000   0.000  1.00  0.00           N
ENDMDL
END
"""

CIF = """\
data_test
#
loop_
_atom_site.group_PDB
_atom_site.id
_atom_site.type_symbol
_atom_site.label_atom_id
_atom_site.label_alt_id
_atom_site.label_comp_id
_atom_site.label_asym_id
_atom_site.label_seq_id
_atom_site.pdbx_PDB_ins_code
_atom_site.Cartn_x
_atom_site.Cartn_y
_atom_site.Cartn_z
_atom_site.occupancy
_atom_site.auth_seq_id
_atom_site.auth_comp_id
_atom_site.auth_asym_id
_atom_site.auth_atom_id
_atom_site.pdbx_PDB_model_num
ATOM   1  N  N   . ALA X 1 ? 0.000 0.000 0.000 1.00 1 ALA A N 1
ATOM   2  C  CA  . ALA X 1 ? 1.458 0.000 0.000 1.00 1 ALA A CA 1
ATOM   3  C  CB  A ALA X 1 ? 1.988 -0.773 1.199 0.40 1 ALA A CB 1
ATOM   4  C  CB  B ALA X 1 ? 1.990 -0.770 1.210 0.60 1 ALA A CB 1
ATOM   5  H  H   . ALA X 1 ? -0.500 0.800 0.000 1.00 1 ALA A H 1
ATOM   6  ?  1HB . ALA X 1 ? 2.500 -0.200 1.900 1.00 1 ALA A 1HB 1
ATOM   7  N  N   . GLY X 2 A 3.300 1.200 -0.500 1.00 1 GLY A N 1
ATOM   8  C  CA  . GLY X 2 A 4.700 1.300 -0.700 1.00 1 GLY A CA 1
HETATM 9  ZN ZN  . ZN  Y . ? 5.000 5.000 5.000 1.00 101 ZN A ZN 1
HETATM 10 O  O   . HOH Z . ? 7.000 7.000 7.000 1.00 201 HOH A O 1
HETATM 11 C  C1  . BTN W . ? 8.000 1.000 2.000 1.00 301 BTN A C1 1
HETATM 12 O  O1  . BTN W . ? 9.000 1.500 2.500 1.00 301 BTN A O1 1
ATOM   13 N  N   . SER V 5 ? 10.000 0.000 0.000 1.00 5 SER B N 1
ATOM   14 O  OG  . SER V 5 ? 11.000 0.500 0.000 1.00 5 SER B OG 1
ATOM   15 N  N   . ALA X 1 ? 50.000 0.000 0.000 1.00 1 ALA A N 2
#
"""


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_pdb_selection_rules(tmp_path):
    from cms_cuda.loader import load_atoms
    p = _write(tmp_path, "t.pdb", PDB)
    xyz, rad, info = load_atoms(p, chains="A")
    assert [(i[2], i[3]) for i in info] == [("ALA", "N"), ("ALA", "CA"), ("ALA", "CB"), ("GLY", "N"), ("GLY", "CA"),
                                            ("BTN", "C1"), ("BTN", "O1")]
    assert np.array_equal(xyz[2], np.float32([1.990, -0.770, 1.210]))   # altloc B (higher occupancy), float32

    assert info[3][:2] == ("A", "1A")                            # insertion code kept in the residue number
    assert (rad > 0).all()
    # keep flags
    _, _, info_w = load_atoms(p, chains="A", keep_water=True, keep_ions=True, keep_hydrogens=True)
    names = [(i[2], i[3]) for i in info_w]
    assert ("HOH", "O") in names and ("ZN", "ZN") in names and ("ALA", "H") in names and ("ALA", "1HB") in names
    # residue-name selection / exclusion, other chain
    _, _, lig = load_atoms(p, resnames={"BTN"})
    assert [i[3] for i in lig] == ["C1", "O1"]
    _, _, nolig = load_atoms(p, chains="A", exclude_resnames={"BTN"})
    assert all(i[2] != "BTN" for i in nolig)
    xb, _, ib = load_atoms(p, chains=["B"])
    assert len(xb) == 2 and ib[0][:3] == ("B", "5", "SER")


def test_mmcif_matches_pdb(tmp_path):
    from cms_cuda.loader import load_atoms
    p = _write(tmp_path, "t.pdb", PDB)
    c = _write(tmp_path, "t.cif", CIF)
    for kw in (dict(chains="A"), dict(chains="B"), dict(resnames={"BTN"}),
               dict(chains="A", keep_water=True, keep_ions=True, keep_hydrogens=True)):
        x1, r1, i1 = load_atoms(p, **kw)
        x2, r2, i2 = load_atoms(c, **kw)
        assert np.array_equal(x1, x2) and np.array_equal(r1, r2)
        assert [(a[0], a[2], a[3]) for a in i1] == [(a[0], a[2], a[3]) for a in i2]


def test_residue_groups_in_first_appearance_order():
    from cms_cuda.loader import residue_groups
    info = [("A", "1", "ALA", "N", "N"), ("A", "1", "ALA", "CA", "C"), ("A", "2", "GLY", "N", "N"),
            ("A", "1", "ALA", "CB", "C")]
    keys, off, atoms = residue_groups(info, first_atom=10)
    assert keys == [("A", "1", "ALA"), ("A", "2", "GLY")]
    assert off.tolist() == [0, 3, 4] and atoms.tolist() == [10, 11, 13, 12]
    keys, off, atoms = residue_groups([])
    assert keys == [] and off.tolist() == [0] and len(atoms) == 0


def test_discontinuous_chain_is_joined_to_its_first_block(tmp_path):
    from cms_cuda.loader import load_atoms
    text = PDB.split("MODEL        2")[0].replace("BTN A 301", "BTN C 301")
    # chain order A, C (ligand), B; then a second block of chain A
    text = text.replace("ENDMDL\n", "ATOM     16  N   ALA A   9      20.000   0.000   0.000  1.00  0.00           N\nENDMDL\n")
    p = _write(tmp_path, "d.pdb", text)
    _, _, info = load_atoms(p, chains="ABC")
    assert [i[0] for i in info] == ["A"] * 6 + ["C"] * 2 + ["B"] * 2
    assert info[5][:2] == ("A", "9")
