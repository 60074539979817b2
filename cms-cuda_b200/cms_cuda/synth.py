"""
Seeded synthetic protein-like complexes (test and benchmark inputs).

Residues are drawn uniformly from the 20 standard amino acids, each with its
standard heavy-atom names; radii come from :func:`get_radii_from_names`.
Coordinates are a self-avoiding random walk with 1.5 A steps that rejects
non-bonded pairs closer than 2.8 A, confined to about 18 cubic A per heavy
atom (``csrc/synth.c``).  Each complex is one such globule cut by a plane of
random orientation into a binder cap and the target; the binder is then slid
out along the plane normal until the closest binder-target pair is 3.5-4.5 A
apart, so the interface spans the whole (complementary) cut.  About 5 % of
batched binders can be small ligand-like clusters with HETATM-style C*/N*/O*
names.
"""

import ctypes
import os

import numpy as np

from .radii import get_radii_from_names, radius_of

_HERE = os.path.dirname(os.path.abspath(__file__))
_SYNTH = os.path.join(_HERE, "libcms_synth.so")

AMINO_ACIDS = {
    "ALA": ("N", "CA", "C", "O", "CB"),
    "ARG": ("N", "CA", "C", "O", "CB", "CG", "CD", "NE", "CZ", "NH1", "NH2"),
    "ASN": ("N", "CA", "C", "O", "CB", "CG", "OD1", "ND2"),
    "ASP": ("N", "CA", "C", "O", "CB", "CG", "OD1", "OD2"),
    "CYS": ("N", "CA", "C", "O", "CB", "SG"),
    "GLN": ("N", "CA", "C", "O", "CB", "CG", "CD", "OE1", "NE2"),
    "GLU": ("N", "CA", "C", "O", "CB", "CG", "CD", "OE1", "OE2"),
    "GLY": ("N", "CA", "C", "O"),
    "HIS": ("N", "CA", "C", "O", "CB", "CG", "ND1", "CD2", "CE1", "NE2"),
    "ILE": ("N", "CA", "C", "O", "CB", "CG1", "CG2", "CD1"),
    "LEU": ("N", "CA", "C", "O", "CB", "CG", "CD1", "CD2"),
    "LYS": ("N", "CA", "C", "O", "CB", "CG", "CD", "CE", "NZ"),
    "MET": ("N", "CA", "C", "O", "CB", "CG", "SD", "CE"),
    "PHE": ("N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "CE1", "CE2", "CZ"),
    "PRO": ("N", "CA", "C", "O", "CB", "CG", "CD"),
    "SER": ("N", "CA", "C", "O", "CB", "OG"),
    "THR": ("N", "CA", "C", "O", "CB", "OG1", "CG2"),
    "TRP": ("N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "NE1", "CE2", "CE3", "CZ2", "CZ3", "CH2"),
    "TYR": ("N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "CE1", "CE2", "CZ", "OH"),
    "VAL": ("N", "CA", "C", "O", "CB", "CG1", "CG2"),
}
_AA = sorted(AMINO_ACIDS)
# radius of every (residue, atom) pair, resolved once
_AA_RADII = {aa: np.array([radius_of(aa, a) for a in AMINO_ACIDS[aa]]) for aa in _AA}
_LIG_RADII = {"C": radius_of("LIG", "C1"), "N": radius_of("LIG", "N1"), "O": radius_of("LIG", "O1")}

STEP, MIN_NB, MIN_FLOOR, VOL_PER_ATOM = 1.5, 2.8, 2.2, 18.0
GAP = (3.5, 4.5)

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_SYNTH):
            raise OSError(f"{_SYNTH} is missing: build it with `python cms-cuda_b200/build.py`")
        lib = ctypes.CDLL(_SYNTH)
        lib.cms_synth_batch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        lib.cms_synth_batch.restype = ctypes.c_int
        _lib = lib
    return _lib


def residue_radii(n_atoms, rng):
    """Radii and (residue, atom) names of n_atoms heavy atoms of random residues."""
    rad, res, atm = [], [], []
    total = 0
    while total < n_atoms:
        aa = _AA[int(rng.integers(len(_AA)))]
        names = AMINO_ACIDS[aa]
        k = min(len(names), n_atoms - total)
        rad.append(_AA_RADII[aa][:k])
        res += [aa] * k
        atm += list(names[:k])
        total += k
    return (np.concatenate(rad) if rad else np.zeros(0)), res, atm


def ligand_radii(n_atoms, rng):
    """HETATM-like ligand cluster: names C*/N*/O* (70/15/15 %)."""
    kinds = rng.choice(np.array(["C", "N", "O"]), size=n_atoms, p=[0.7, 0.15, 0.15])
    rad = np.array([_LIG_RADII[k] for k in kinds])
    return rad, ["LIG"] * n_atoms, [f"{k}{i + 1}" for i, k in enumerate(kinds)]


class Batch:
    """Concatenated batch: binder atoms then target atoms per complex."""

    def __init__(self, atom_off, n_binder, xyz, radius, gaps=None, ligand=None, names=None):
        self.names = names          # optional (residue names, atom names, residue numbers) per atom
        self.atom_off = np.asarray(atom_off, dtype=np.int64)
        self.n_binder = np.asarray(n_binder, dtype=np.int64)
        self.xyz = xyz
        self.radius = radius
        self.gaps = gaps
        self.ligand = ligand if ligand is not None else np.zeros(len(self.n_binder), bool)

    @property
    def B(self):
        return len(self.n_binder)

    @property
    def N(self):
        return int(self.atom_off[-1])

    def complex(self, c):
        """(binder_xyz, binder_radii, target_xyz, target_radii) of complex c."""
        a0, a1 = self.atom_off[c], self.atom_off[c + 1]
        s1 = a0 + self.n_binder[c]
        return self.xyz[a0:s1], self.radius[a0:s1], self.xyz[s1:a1], self.radius[s1:a1]


def make_batch(n_target, n_binder, seed, ligand=None, threads=None, names=False, select=None):
    """
    Generate a batch of complexes with the given per-complex atom counts.
    ligand: optional bool array marking binders that are ligand clusters.
    names: also keep each atom's residue name, atom name and residue number.
    select: optional complex indices; only those complexes are generated (in
    that order), each identical to its copy in the full batch.
    """
    n_target = np.asarray(n_target, dtype=np.int32).reshape(-1)
    n_binder = np.asarray(n_binder, dtype=np.int32).reshape(-1)
    B = len(n_target)
    ligand = np.zeros(B, bool) if ligand is None else np.asarray(ligand, bool)
    rng = np.random.default_rng(seed)
    seeds = rng.integers(0, 2**63 - 1, size=B, dtype=np.int64).astype(np.uint64)
    if select is not None:
        select = np.asarray(select, dtype=np.int64)
        n_target, n_binder, ligand, seeds = n_target[select], n_binder[select], ligand[select], seeds[select]
        B = len(select)
    atom_off = np.zeros(B + 1, dtype=np.int64)
    atom_off[1:] = np.cumsum(n_target.astype(np.int64) + n_binder)
    N = int(atom_off[-1])
    xyz = np.empty((N, 3))
    perm = np.empty(N, dtype=np.int32)
    gaps = np.empty(B)
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    st = _load().cms_synth_batch(B, n_target.ctypes.data, n_binder.ctypes.data, seeds.ctypes.data,
                                 atom_off.ctypes.data, STEP, MIN_NB, MIN_FLOOR, VOL_PER_ATOM, GAP[0], GAP[1],
                                 xyz.ctypes.data, perm.ctypes.data, gaps.ctypes.data)
    if st != 0:
        raise RuntimeError("synthetic generator failed")
    radius = np.empty(N)
    res_n = np.empty(N, dtype=object) if names else None
    atm_n = np.empty(N, dtype=object) if names else None
    res_i = np.empty(N, dtype=np.int64) if names else None
    for c in range(B):
        crng = np.random.default_rng(int(seeds[c]) ^ 0x5EED)
        a0, a1 = int(atom_off[c]), int(atom_off[c + 1])
        nb = int(n_binder[c])
        walk_r, wres, watm = residue_radii(a1 - a0, crng)        # radii and names along the walk
        p = perm[a0:a1]
        radius[a0:a1] = walk_r[p]
        if names:
            starts = np.r_[True, np.array(wres[1:], dtype=object) != np.array(wres[:-1], dtype=object)] \
                if len(wres) else np.zeros(0, bool)
            first = [i for i in range(len(watm)) if i == 0 or watm[i] == "N" or starts[i]]
            rid = np.zeros(len(watm), np.int64)
            for k, f in enumerate(first):
                rid[f:] = k + 1
            res_n[a0:a1] = np.array(wres, dtype=object)[p]
            atm_n[a0:a1] = np.array(watm, dtype=object)[p]
            res_i[a0:a1] = rid[p]
        if ligand[c]:
            lr, lres, latm = ligand_radii(nb, crng)
            radius[a0:a0 + nb] = lr
            if names:
                res_n[a0:a0 + nb] = lres
                atm_n[a0:a0 + nb] = latm
                res_i[a0:a0 + nb] = 1
    return Batch(atom_off, n_binder, xyz, radius, gaps, ligand, (res_n, atm_n, res_i) if names else None)


def write_pdb(path, batch, c, binder_chain="B", target_chain="A"):
    """Write complex c of a batch made with names=True as a PDB file (binder and target chains)."""
    res_n, atm_n, res_i = batch.names
    a0, a1 = int(batch.atom_off[c]), int(batch.atom_off[c + 1])
    s1 = a0 + int(batch.n_binder[c])
    with open(path, "w") as f:
        serial = 1
        for lo, hi, ch in ((a0, s1, binder_chain), (s1, a1, target_chain)):
            for g in range(lo, hi):
                nm = str(atm_n[g])
                name = nm if len(nm) == 4 else " " + nm.ljust(3)
                rec = "HETATM" if res_n[g] == "LIG" else "ATOM  "
                x, y, z = batch.xyz[g]
                el = nm.lstrip("0123456789")[:1]
                f.write(f"{rec}{serial:5d} {name}{'':1}{res_n[g]:>3s} {ch}{int(res_i[g]):4d}    "
                        f"{x:8.3f}{y:8.3f}{z:8.3f}{1.0:6.2f}{0.0:6.2f}          {el:>2s}\n")
                serial += 1
            f.write("TER\n")
        f.write("END\n")


def make_complex(n_target, n_binder, seed):
    """One complex: (binder_xyz, binder_radii, target_xyz, target_radii)."""
    return make_batch([n_target], [n_binder], seed).complex(0)


def config_plain_small(seed=0):
    """Target 1200 heavy atoms, binder 450."""
    return make_complex(1200, 450, seed)


def config_plain_large(seed=1):
    """Antibody-sized target 8000 heavy atoms, binder 1800."""
    return make_complex(8000, 1800, seed)


def config_refine(B=256, seed=5):
    """Pose-refinement batch: target uniform 1500-3000, binder uniform 300-800 atoms."""
    rng = np.random.default_rng(seed)
    nt = rng.integers(1500, 3001, B).astype(np.int32)
    nb = rng.integers(300, 801, B).astype(np.int32)
    return make_batch(nt, nb, seed + 1)


def batched_sizes(B=4096, seed=2):
    """(target atoms, binder atoms, ligand flag) per complex of config_batched(B, seed), without the coordinates."""
    rng = np.random.default_rng(seed)
    nt = np.exp(rng.uniform(np.log(600), np.log(4000), B)).astype(np.int32)
    nb = np.exp(rng.uniform(np.log(80), np.log(1200), B)).astype(np.int32)
    lig = rng.random(B) < 0.05
    nb[lig] = rng.integers(20, 61, int(lig.sum()))
    return nt, nb, lig


def config_batched(B=4096, seed=2, select=None):
    """
    B complexes, target log-uniform 600-4000, binder log-uniform 80-1200, ~5 %
    ligand binders of 20-60 atoms; `select` generates only those complexes
    (a shard of the batch).
    """
    nt, nb, lig = batched_sizes(B, seed)
    return make_batch(nt, nb, seed + 1, ligand=lig, select=select)
