"""
Heavy-atom loader for PDB and mmCIF files with the reference CLI's selection
rules (examples/calculate_cms_sc.py:43-97), without a Biopython dependency.

One side of an interface is selected by chain IDs and/or residue names:

* first model only (NMR / multi-model files);
* one alternate location per atom: the highest occupancy, the first on ties;
* water (HOH, WAT, DOD, H2O, TIP, TIP3, SOL, or a HETATM water) dropped unless
  keep_water; single-atom HETATM residues (ions) dropped unless keep_ions;
* hydrogens dropped unless keep_hydrogens: element H or D, or, without an
  element, an atom name starting with H or D after leading digits;
* radii from get_radii_from_names (0 for names without a table entry).

Returns xyz (N, 3) float64, radii (N,) float64 and one (chain, residue number
+ insertion code, residue name, atom name, element) tuple per atom -- the
reference loader's outputs, in its order and with its coordinate rounding: the
reference reads structures with Biopython, which groups atoms by chain (chains
in order of first appearance, a discontinuous chain joined to its first
block), residues in order of first appearance within the chain, and stores
coordinates as float32, so each coordinate here is the float32 nearest to the
file's decimal, widened to float64.
"""

import shlex

import numpy as np

from .radii import get_radii_from_names

WATER_NAMES = {"HOH", "WAT", "DOD", "H2O", "TIP", "TIP3", "SOL"}


def _is_hydrogen(name, element):
    return element in ("H", "D") or (element in ("", "X") and name.lstrip("0123456789").startswith(("H", "D")))


def _records_pdb(path):
    """Atom records of the first model: dicts with the fields the selection needs."""
    out = []
    with open(path) as fh:
        for line in fh:
            rec = line[:6]
            if rec.startswith("ENDMDL"):
                break
            if not (rec.startswith("ATOM") or rec.startswith("HETATM")):
                continue
            name = line[12:16].strip()
            element = line[76:78].strip().upper() if len(line) >= 78 else ""
            try:
                occ = float(line[54:60])
            except ValueError:
                occ = 1.0
            out.append(dict(het=rec.startswith("HETATM"), name=name, alt=line[16:17].strip(),
                            resn=line[17:20].strip(), chain=line[21:22].strip(), resseq=line[22:26].strip(),
                            icode=line[26:27].strip(), x=float(line[30:38]), y=float(line[38:46]),
                            z=float(line[46:54]), occ=occ, element=element))
    return out


def _cif_tokens(lines):
    for line in lines:
        if line.startswith(";"):
            continue
        for t in shlex.split(line, posix=True):
            yield t


def _records_cif(path):
    """Atom records of the first model from the _atom_site loop."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    i = 0
    while i < len(lines):
        if lines[i].strip() == "loop_" and i + 1 < len(lines) and lines[i + 1].strip().startswith("_atom_site."):
            break
        i += 1
    else:
        return []
    i += 1
    cols = []
    while i < len(lines) and lines[i].strip().startswith("_atom_site."):
        cols.append(lines[i].strip().split(".", 1)[1].split()[0])
        i += 1
    body = []
    while i < len(lines):
        s = lines[i].strip()
        if s.startswith("#") or s.startswith("loop_") or s.startswith("_") or s.startswith("data_"):
            break
        if s:
            body.append(lines[i])
        i += 1
    toks = list(_cif_tokens(body))
    n = len(cols)
    col = {c: k for k, c in enumerate(cols)}

    def get(row, *names, default=""):
        for nm in names:
            k = col.get(nm)
            if k is not None:
                v = row[k]
                return "" if v in ("?", ".") else v
        return default

    out, model0 = [], None
    for r in range(0, len(toks) - n + 1, n):
        row = toks[r:r + n]
        model = get(row, "pdbx_PDB_model_num")
        if model0 is None:
            model0 = model
        elif model != model0:
            break
        occ = get(row, "occupancy")
        out.append(dict(het=get(row, "group_PDB") == "HETATM",
                        name=get(row, "auth_atom_id", "label_atom_id"),
                        alt=get(row, "label_alt_id"),
                        resn=get(row, "auth_comp_id", "label_comp_id"),
                        chain=get(row, "auth_asym_id", "label_asym_id"),
                        resseq=get(row, "auth_seq_id", "label_seq_id"),
                        icode=get(row, "pdbx_PDB_ins_code"),
                        x=float(get(row, "Cartn_x")), y=float(get(row, "Cartn_y")), z=float(get(row, "Cartn_z")),
                        occ=float(occ) if occ else 1.0,
                        element=get(row, "type_symbol").upper()))
    return out


def read_records(path):
    p = str(path).lower()
    return _records_cif(path) if p.endswith((".cif", ".mmcif")) else _records_pdb(path)


def load_atoms(path, chains=None, resnames=None, exclude_resnames=(), keep_water=False, keep_ions=False,
               keep_hydrogens=False):
    """Heavy atoms of one side of an interface: (xyz, radii, info)."""
    if isinstance(chains, str):
        chains = [c for c in chains.split(",") if c] if "," in chains else list(chains)
    recs = read_records(path)
    # residues grouped by chain, atoms per residue (alternate locations resolved)
    residues = {}
    chain_res = {}
    for rc in recs:
        key = (rc["chain"], rc["het"], rc["resseq"], rc["icode"], rc["resn"])
        if key not in residues:
            residues[key] = {"het": rc["het"], "atoms": {}, "order": []}
            chain_res.setdefault(rc["chain"], []).append(key)
        res = residues[key]
        atoms = res["atoms"]
        if rc["name"] in atoms:
            if rc["occ"] > atoms[rc["name"]]["occ"]:           # highest occupancy, first on ties
                atoms[rc["name"]] = rc
        else:
            atoms[rc["name"]] = rc
            res["order"].append(rc["name"])
    xyz, res_names, atom_names, info = [], [], [], []
    for key in (k for keys in chain_res.values() for k in keys):
        chain, _, resseq, icode, resn = key
        res = residues[key]
        if chains is not None and chain not in chains:
            continue
        if resnames is not None and resn not in resnames:
            continue
        if resn in exclude_resnames:
            continue
        if not keep_water and resn in WATER_NAMES:
            continue
        if not keep_ions and res["het"] and len(res["order"]) == 1:
            continue
        for nm in res["order"]:
            a = res["atoms"][nm]
            if not keep_hydrogens and _is_hydrogen(nm, a["element"]):
                continue
            xyz.append((a["x"], a["y"], a["z"]))
            res_names.append(resn)
            atom_names.append(nm)
            info.append((chain, f"{resseq}{icode}", resn, nm, a["element"]))
    xyz = np.asarray(xyz, dtype=np.float32).astype(np.float64).reshape(-1, 3)
    return xyz, get_radii_from_names(res_names, atom_names), info


def residue_groups(info, first_atom=0):
    """
    Residues of one side as a CSR map for the device's per-residue sums
    (``Context.residue_sums``): the residue keys (chain, residue number, residue
    name) in order of first appearance, offsets (len(keys) + 1, int64) and the
    member atoms of each residue in atom order (int32), shifted by
    ``first_atom`` -- the side's first atom in a batch.  The reference CLI keys
    its per-residue table the same way (examples/calculate_cms_sc.py:105-114).
    """
    slot = {}
    member = np.empty(len(info), dtype=np.int64)
    for a, rec in enumerate(info):
        member[a] = slot.setdefault(rec[:3], len(slot))
    keys = list(slot)
    atoms = np.argsort(member, kind="stable").astype(np.int32) + np.int32(first_atom)
    off = np.zeros(len(keys) + 1, dtype=np.int64)
    np.cumsum(np.bincount(member, minlength=len(keys)), out=off[1:])
    return keys, off, atoms
