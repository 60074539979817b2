"""
Minimal fixed-column PDB reader: heavy atoms of selected chains, with radii.

It mirrors the atom selection the reference uses around the hot path
(test/test_gpu_parity.py:52-69 and examples/calculate_cms_sc.py:43-97):
ATOM and HETATM records of the first model, hydrogens dropped (element ``H``,
a name starting with ``H``, or a digit followed by ``H`` such as ``1HB``),
radii from :func:`cms_cuda.get_radii_from_names`.  Alternate locations keep the
first one seen for each atom.
"""

import numpy as np

from .radii import get_radii_from_names


def _is_hydrogen(name, element):
    return (element == "H" or name.startswith("H")
            or (len(name) > 1 and name[0].isdigit() and name[1] == "H"))


def read_pdb_chains(path):
    """Parse a PDB file into {chain: (xyz (N,3) f64, res_names, atom_names)}."""
    chains = {}
    seen = set()
    with open(path) as fh:
        for line in fh:
            rec = line[:6]
            if rec.startswith("ENDMDL"):
                break
            if not (rec.startswith("ATOM") or rec.startswith("HETATM")):
                continue
            name = line[12:16].strip()
            alt = line[16:17]
            resn = line[17:20].strip()
            chain = line[21:22]
            resi = line[22:27]
            element = line[76:78].strip().upper() if len(line) >= 78 else ""
            if not element:
                element = "".join(c for c in name if c.isalpha())[:1].upper()
            if _is_hydrogen(name, element):
                continue
            key = (chain, resi, resn, name)
            if alt.strip() and key in seen:
                continue
            seen.add(key)
            x, y, z = float(line[30:38]), float(line[38:46]), float(line[46:54])
            c = chains.setdefault(chain, ([], [], []))
            c[0].append((x, y, z))
            c[1].append(resn)
            c[2].append(name)
    return {k: (np.asarray(v[0], dtype=np.float64).reshape(-1, 3), v[1], v[2])
            for k, v in chains.items()}


def load_complex(path, binder_chains="B", target_chains="A"):
    """
    (binder_xyz, binder_radii, target_xyz, target_radii) from a PDB file.
    Chain B is the binder and chain A the target by default, as in the
    reference's parity test.
    """
    ch = read_pdb_chains(path)

    def side(ids):
        xyz, res, atm = [], [], []
        for c in ids:
            if c in ch:
                xyz.append(ch[c][0]); res += ch[c][1]; atm += ch[c][2]
        xyz = np.concatenate(xyz) if xyz else np.zeros((0, 3))
        return xyz, get_radii_from_names(res, atm), res, atm

    bx, br, _, _ = side(binder_chains)
    tx, tr, _, _ = side(target_chains)
    return bx, br, tx, tr
