"""
Atomic radii for contact molecular surface / shape complementarity.

The table is the Rosetta shape-complementarity radii library that the
reference ships as ``SC_RADII_LIB`` (cms-cuda/_core.py:172-269); the numbers
must be identical because CMS is only meaningful with these radii.  The lookup
follows ``get_radii_from_names`` / ``wildcard_match`` (_core.py:87-112,
719-758): the first table row whose residue pattern and atom pattern both
match wins, ``*`` in a pattern matches the rest of the name, and an unmatched
atom gets radius 0.

Matching is memoised per distinct (residue, atom) pair, so a batch of millions
of atoms costs one table scan per distinct name pair instead of one per atom.
"""

import functools

import numpy as np

# (residue pattern, atom pattern, radius) in table order -- order matters:
# the first match wins.
_TABLE = (
    ("ALA", "CB", 1.95), ("ARG", "NH*", 1.70), ("ARG", "CZ", 1.80), ("ARG", "NE", 1.65),
    ("ARG", "CD", 1.90), ("ARG", "CG", 1.90), ("ASN", "ND2", 1.70), ("ASN", "OD1", 1.60),
    ("ASN", "CG", 1.80), ("ASP", "OD*", 1.60), ("ASP", "CG", 1.80), ("GLN", "NE2", 1.70),
    ("GLN", "OE1", 1.60), ("GLN", "CD", 1.80), ("GLN", "CG", 1.90), ("GLU", "OE*", 1.60),
    ("GLU", "CD", 1.80), ("GLU", "CG", 1.90), ("GLY", "CA", 1.90), ("HIS", "CD2", 1.90),
    ("HIS", "NE2", 1.65), ("HIS", "CE1", 1.90), ("HIS", "ND1", 1.65), ("HIS", "CG", 1.80),
    ("HOH", "O*", 1.70), ("ILE", "CD1", 1.95), ("ILE", "CG1", 1.90), ("ILE", "CB", 1.85),
    ("ILE", "CG2", 1.95), ("LEU", "CD*", 1.95), ("LEU", "CG", 1.85), ("LYS", "NZ", 1.75),
    ("LYS", "CE", 1.90), ("LYS", "CD", 1.90), ("LYS", "CG", 1.90), ("MET", "CE", 1.95),
    ("MET", "CG", 1.90), ("PHE", "CD*", 1.90), ("PHE", "CE*", 1.90), ("PHE", "CZ", 1.90),
    ("PHE", "CG", 1.80), ("PRO", "CD", 1.90), ("PRO", "CG", 1.90), ("SER", "OG", 1.70),
    ("SUL", "S", 1.90), ("SUL", "O*", 1.65), ("THR", "CG2", 1.95), ("THR", "OG1", 1.70),
    ("THR", "CB", 1.85), ("TRP", "CE2", 1.80), ("TRP", "CE3", 1.90), ("TRP", "CD1", 1.90),
    ("TRP", "CD2", 1.80), ("TRP", "CZ*", 1.90), ("TRP", "CH2", 1.90), ("TRP", "NE1", 1.65),
    ("TRP", "CG", 1.80), ("TYR", "OH", 1.70), ("TYR", "CD*", 1.90), ("TYR", "CE*", 1.90),
    ("TYR", "CZ", 1.80), ("TYR", "CG", 1.80), ("VAL", "CG*", 1.95), ("VAL", "CB", 1.85),
    ("WAT", "O", 1.70), ("WAT", "O*", 1.70), ("LG*", "HARO", 1.00), ("LG*", "AROC", 2.00),
    ("LG*", "ARO", 2.00), ("LG*", "NHIS", 1.75), ("LG*", "NHI", 1.75), ("LG*", "COO", 1.55),
    ("LG*", "OCBB", 1.55), ("LG*", "OCB", 1.55), ("LG*", "OOC", 1.55), ("LG*", "NLYS", 1.75),
    ("*", "H", 0.50), ("*", "H*", 0.50), ("*", "1H*", 0.50), ("*", "2H*", 0.50),
    ("*", "3H*", 0.50), ("*", "C", 1.80), ("*", "CA", 1.85), ("*", "CB", 1.90),
    ("*", "C*", 1.85), ("*", "N", 1.65), ("*", "N*", 1.65), ("*", "O", 1.60),
    ("*", "O*", 1.60), ("*", "OXT", 1.60), ("*", "OT*", 1.60), ("*", "S*", 1.90),
    ("*", "P", 2.15), ("*", "P*", 2.15), ("*", "F*", 1.50),
)


def wildcard_match(query, pattern, limit):
    """
    Character-by-character match of a stripped name against a table pattern,
    comparing at most ``limit - 1`` positions (the reference passes
    ``len(query) + 2``).  Past the end of a string its character reads as NUL;
    ``*`` matches anything and, when it is the pattern's last character, ends
    the match successfully; a query space matches the end of the pattern.
    Same semantics as _core.py:719-758.
    """
    qi = pi = 0
    nq, np_ = len(query), len(pattern)
    while True:
        limit -= 1
        if limit <= 0:
            return True
        q = query[qi] if qi < nq else "\0"
        p = pattern[pi] if pi < np_ else "\0"
        if not (q == p or p == "*" or (q == " " and p == "\0")):
            return False
        if p == "*" and (pi + 1 >= np_ or pattern[pi + 1] == "\0"):
            return True
        if q != "\0":
            qi += 1
        if p != "\0":
            pi += 1


@functools.lru_cache(maxsize=65536)
def radius_of(res, atom):
    """Radius of one (residue name, atom name) pair; 0.0 when nothing matches."""
    for rpat, apat, rad in _TABLE:
        if wildcard_match(res, rpat, len(res) + 2) and wildcard_match(atom, apat, len(atom) + 2):
            return rad
    return 0.0


def get_radii_from_names(res_names, atom_names):
    """
    Radii for parallel lists of stripped residue and atom names
    (the reference's ``get_radii_from_names``, _core.py:87-112).

    Returns float64 array of shape (N,), 0.0 for unmatched atoms.
    """
    res_names = list(res_names)
    atom_names = list(atom_names)
    if len(res_names) != len(atom_names):
        raise ValueError("res_names and atom_names must have the same length")
    out = np.zeros(len(res_names), dtype=np.float64)
    for i, (r, a) in enumerate(zip(res_names, atom_names)):
        out[i] = radius_of(str(r), str(a))
    return out
