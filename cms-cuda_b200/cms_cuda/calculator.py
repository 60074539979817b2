"""
Drop-in ``MolecularSurfaceCalculator`` backed by the B200 CUDA library.

Same settings, methods, return types, caching and errors as the reference
calculator (cms-cuda/_core.py:762-1147; its GPU twin cms-cuda/_gpu.py:310-686):

* ``settings`` (rp, density, band, sep, weight, binwidth_dist, binwidth_norm);
  density is stored per atom when ``AddMolecule`` is called;
* ``reset``, ``add_binder_and_target``, ``AddMolecule``;
* ``CalcLoaded``, ``CalcLoadedSC``, ``CalcLoadedMaxPossibleCMS``,
  ``calc_contact_molecular_surface(target_side)``;
* ``run`` -- the same containers the reference fills (results, atoms, dots,
  trimmed_dots, probes, neighbor_array, buried_array, toroid_queue, radmax,
  surfaces_generated[_all_atoms]), copied from the device lazily on first
  access instead of after every generation.

All arithmetic runs on the GPU; nothing falls back to the CPU.
"""

import numpy as np

from . import _lib


ATTEN_BLOCKER = 1
ATTEN_2 = 2
ATTEN_BURIED_FLAGGED = 5
ATTEN_6 = 6
MAX_SUBDIV = 100


class _Obj:
    pass


class ResultsSurface:
    def __init__(self):
        self.d_mean = 0.0
        self.d_median = 0.0
        self.s_mean = 0.0
        self.s_median = 0.0
        self.nAtoms = 0
        self.nBuriedAtoms = 0
        self.nBlockedAtoms = 0
        self.nAllDots = 0
        self.nTrimmedDots = 0
        self.nBuriedDots = 0
        self.nAccessibleDots = 0
        self.trimmedArea = 0.0


class ResultsDots:
    def __init__(self):
        self.convex = 0
        self.concave = 0
        self.toroidal = 0


class RESULTS:
    def __init__(self):
        self.sc = 0.0
        self.area = 0.0
        self.distance = 0.0
        self.perimeter = 0.0
        self.nAtoms = 0
        self.surface = [ResultsSurface(), ResultsSurface(), ResultsSurface()]
        self.dots = ResultsDots()
        self.valid = 0


class AtomArray:
    """Struct of arrays of the loaded atoms (the reference's AtomArray fields)."""

    def __init__(self, n=0):
        self.xyz = np.zeros((n, 3))
        self.radius = np.zeros(n)
        self.density = np.zeros(n)
        self.molecule = np.zeros(n, np.int8)
        self.atten = np.zeros(n, np.int8)
        self.access = np.zeros(n, np.int8)
        self.natom = np.arange(n, dtype=np.int32)
        self.nresidue = np.zeros(n, np.int32)
        self.atom_name = [''] * n
        self.residue_name = [''] * n

    def __len__(self):
        return len(self.radius)

    def __bool__(self):
        return len(self.radius) > 0


class DotArray:
    """Struct of arrays of one molecule's dots (the reference's DotArray fields)."""

    def __init__(self):
        self.coor_xyz = np.zeros((0, 3))
        self.outnml_xyz = np.zeros((0, 3))
        self.area = np.zeros(0)
        self.buried = np.zeros(0, np.int8)
        self.type_ = np.zeros(0, np.int8)
        self.atom_idx = np.zeros(0, np.int32)

    def __len__(self):
        return len(self.area)

    def __bool__(self):
        return len(self.area) > 0


class ProbeArray:
    def __init__(self):
        self.height = np.zeros(0)
        self.atom_idx_0 = np.zeros(0, np.int32)
        self.atom_idx_1 = np.zeros(0, np.int32)
        self.atom_idx_2 = np.zeros(0, np.int32)
        self.point_xyz = np.zeros((0, 3))
        self.alt_xyz = np.zeros((0, 3))

    def __len__(self):
        return len(self.height)

    def __bool__(self):
        return len(self.height) > 0


class SimpleNeighborArray:
    """Padded (N, K) neighbour table: NaN / -1 padding, K = longest row (>= 1)."""

    def __init__(self, cap, max_neighbors):
        self._cap = cap
        self._max_neighbors = max_neighbors
        self.xyz = np.full((cap, max_neighbors, 3), np.nan)
        self.radius = np.full((cap, max_neighbors), np.nan)
        self.natom = np.full((cap, max_neighbors), -1, dtype=np.int32)
        self.nneighbors = np.zeros(cap, dtype=np.int32)

    def __len__(self):
        return self._cap

    def __bool__(self):
        return self._cap > 0


class _Lease:
    """
    A pooled library context borrowed for one generated surface.  The
    calculator and its ``run`` both hold the lease; the context goes back to
    the pool when neither needs it any more.
    """

    def __init__(self, device):
        self.device = device
        self.ctx = _lib.acquire_context(device)

    def __del__(self):
        try:
            _lib.release_context(self.ctx, self.device)
        except Exception:
            pass


class _Run:
    """``calc.run``; device state is copied into host containers on first access."""

    _LAZY = ("atoms", "dots", "trimmed_dots", "probes", "neighbor_array", "buried_array", "toroid_queue")

    def __init__(self):
        self.radmax = 0.0
        self.results = RESULTS()
        self._host = {}
        self._state = None          # (lease, inputs, n, n0, sc_done, order) once a surface exists
        self.surfaces_generated = False
        self.surfaces_generated_all_atoms = None

    def __getattr__(self, name):
        if name in _Run._LAZY:
            host = self.__dict__["_host"]
            if name not in host:
                st = self.__dict__.get("_state")
                host[name] = _export(self, st, name) if st is not None else _Run._empty(name)
            return host[name]
        raise AttributeError(name)

    @staticmethod
    def _empty(name):
        return {"atoms": AtomArray(0), "dots": [DotArray(), DotArray()], "trimmed_dots": [DotArray(), DotArray()],
                "probes": ProbeArray(), "neighbor_array": None, "buried_array": None, "toroid_queue": []}[name]


def _export(run, st, name):
    """
    Host copy of one calc.run container from the device state of the run's
    surface.  The device holds the atoms binder first; `order` (None when the
    atoms were added binder first) maps each device position to the atom's
    position in AddMolecule order, the reference's natom numbering
    (_core.py:372-399), and every container is returned in that numbering.
    """
    lease, (xyz, rad, dens, mol), n, n0, sc_done, order = st
    ctx = lease.ctx

    def user(idx):
        return idx if order is None else order[idx].astype(np.int32)

    def rows_by_atom(atom_of_row):
        # rows are grouped by generating atom in device order; the reference groups them in natom order
        return slice(None) if order is None else np.argsort(order[atom_of_row], kind="stable")

    if name == "atoms":
        a = AtomArray(n)
        atten, access, _, _ = ctx.export_atoms(0, n)
        if order is not None:          # device order -> AddMolecule order (the inputs are kept in that order)
            atten_d, access_d = atten, access
            atten, access = np.empty_like(atten_d), np.empty_like(access_d)
            atten[order], access[order] = atten_d, access_d
        a.xyz, a.radius, a.density, a.molecule, a.atten, a.access = xyz, rad, dens, mol, atten, access
        return a
    info = ctx.info(0)
    if name in ("neighbor_array", "buried_array"):
        nb_off, nb_id, bu_off, bu_id = ctx.export_neighbors(0, n, info)
        off, ids = (nb_off, nb_id) if name == "neighbor_array" else (bu_off, bu_id)
        cnt = np.diff(off).astype(np.int32)
        K = max(int(cnt.max()) if len(cnt) and cnt.any() else 1, 1)
        arr = SimpleNeighborArray(n, K)
        rows = np.repeat(np.arange(n), cnt)
        cols = np.arange(len(ids)) - np.repeat(off[:-1], cnt)
        ids = user(ids)
        if order is not None:
            rows = order[rows]
        arr.natom[rows, cols] = ids
        arr.radius[rows, cols] = rad[ids]
        arr.xyz[rows, cols] = xyz[ids]
        arr.nneighbors[np.arange(n) if order is None else order] = cnt
        return arr
    if name == "toroid_queue":
        a1, a2, uij, tij, rij, bet = ctx.export_toroid(0, info)
        k = rows_by_atom(a1)
        a1, a2, uij, tij, rij, bet = user(a1)[k], user(a2)[k], uij[k], tij[k], rij[k], bet[k]
        return [(int(a1[k]), int(a2[k]), uij[k], tij[k], float(rij[k]), bool(bet[k])) for k in range(len(a1))]
    if name == "probes":
        a0, a1, a2, h, pt, alt = ctx.export_probes(0, info)
        if order is not None:
            # all '+' probes (atoms i, j, k), then all '-' probes (atoms j, i, k), each in natom order of i
            npl = int(info.n_probes_plus[0] + info.n_probes_plus[1])
            k = np.concatenate([rows_by_atom(a0[:npl]), npl + rows_by_atom(a1[npl:])])
            a0, a1, a2, h, pt, alt = user(a0)[k], user(a1)[k], user(a2)[k], h[k], pt[k], alt[k]
        p = ProbeArray()
        p.atom_idx_0, p.atom_idx_1, p.atom_idx_2, p.height, p.point_xyz, p.alt_xyz = a0, a1, a2, h, pt, alt
        return p
    if name == "dots":
        out = []
        for m in (0, 1):
            d = DotArray()
            d.coor_xyz, d.outnml_xyz, d.area, d.buried, d.type_, d.atom_idx = ctx.export_dots(0, m, info)
            d.atom_idx = user(d.atom_idx)
            out.append(d)
        return out
    if name == "trimmed_dots":
        if not sc_done[0]:
            return [DotArray(), DotArray()]
        dots = run.dots
        out = []
        for m in (0, 1):
            idx = ctx.export_trimmed(0, m, info)
            src = dots[m]
            t = DotArray()
            t.coor_xyz, t.outnml_xyz, t.area = src.coor_xyz[idx], src.outnml_xyz[idx], src.area[idx]
            t.buried, t.type_, t.atom_idx = src.buried[idx], src.type_[idx], src.atom_idx[idx]
            out.append(t)
        return out
    raise AttributeError(name)


class MolecularSurfaceCalculator:

    def __init__(self, device=0):
        self.settings = type("Settings", (), {})()
        self.settings.rp = 1.7
        self.settings.density = 15.0
        self.settings.band = 1.5
        self.settings.sep = 8.0
        self.settings.weight = 0.5
        self.settings.binwidth_dist = 0.02
        self.settings.binwidth_norm = 0.02
        self._device = device
        self.reset()

    # -- loading ---------------------------------------------------------------
    def reset(self):
        # a previous run keeps its own lease (and so its device state)
        self.run = _Run()
        self._lease = None
        self._xyz = []
        self._rad = []
        self._dens = []
        self._mol = []
        self._cms = None
        self._sc = None
        self._max = None

    def add_binder_and_target(self, binder_xyz, binder_radii, target_xyz, target_radii):
        self.reset()
        self.AddMolecule(0, binder_xyz, binder_radii)
        self.AddMolecule(1, target_xyz, target_radii)

    def AddMolecule(self, molecule, xyz, radii):
        """
        Load atoms of one molecule (0 = binder, anything else = target), in
        any order and any number of calls (_core.py:923-943).  Atoms with
        radius <= 0 are kept so per-atom outputs stay aligned.  Atoms are
        numbered in call order (calc.run uses that numbering); per-atom
        readouts list one molecule's atoms in the order they were added.
        """
        if hasattr(xyz, "detach"):
            xyz = xyz.detach().cpu().numpy()
        if hasattr(radii, "detach"):
            radii = radii.detach().cpu().numpy()
        mol = 1 if molecule == 1 else 0
        radii = np.asarray(radii, dtype=np.float64).reshape(-1)
        n = len(radii)
        xyz = np.asarray(xyz, dtype=np.float64).reshape(n, 3) if n else np.zeros((0, 3))
        if n == 0:
            return
        self._xyz.append(xyz.copy())
        self._rad.append(radii.copy())
        self._dens.append(np.full(n, float(self.settings.density)))
        self._mol.append(mol)
        self.run.results.surface[mol].nAtoms += n
        self.run.results.nAtoms += n

    def _arrays(self):
        """Atoms in AddMolecule order, and the device order: binder atoms first, each molecule in call order."""
        xyz = np.concatenate(self._xyz) if self._xyz else np.zeros((0, 3))
        rad = np.concatenate(self._rad) if self._rad else np.zeros(0)
        dens = np.concatenate(self._dens) if self._dens else np.zeros(0)
        mol = np.concatenate([np.full(len(r), m, np.int8) for r, m in zip(self._rad, self._mol)]) \
            if self._rad else np.zeros(0, np.int8)
        order = np.argsort(mol, kind="stable")
        if np.all(mol[:-1] <= mol[1:]):
            order = None
        return xyz, rad, dens, mol, order

    # -- generation --------------------------------------------------------------
    def _context(self):
        if self._lease is None:
            self._lease = _Lease(self._device)
        return self._lease.ctx

    def _ensure_surfaces_generated(self, all_atoms=False):
        if self.run.surfaces_generated:
            if self.run.surfaces_generated_all_atoms != all_atoms:
                raise RuntimeError(
                    "This MolecularSurfaceCalculator instance already generated its "
                    f"molecular surface with all_atoms={self.run.surfaces_generated_all_atoms}, "
                    f"but was asked to reuse it with all_atoms={all_atoms}. These use "
                    "incompatible attention-number assignments (CalcLoadedMaxPossibleCMS's "
                    "all_atoms=True vs. CalcLoaded()/CalcLoadedSC()'s all_atoms=False), so "
                    "the cached surface can't be safely reused for both. Call self.reset() "
                    "and re-add your atoms, or use a fresh MolecularSurfaceCalculator()."
                )
            return
        xyz, rad, dens, mol, order = self._arrays()
        assert len(rad) > 0
        ctx = self._context()
        ctx.set_settings(self.settings)
        n0 = int((mol == 0).sum())
        if order is None:
            ctx.load_batch(np.array([0, len(rad)]), np.array([n0]), xyz, rad, dens)
        else:
            ctx.load_batch(np.array([0, len(rad)]), np.array([n0]), xyz[order], rad[order], dens[order])
        ctx.generate(all_atoms=all_atoms)
        info = ctx.info(0)
        if info.status & _lib.ST_COINCIDENT:
            i, j = info.coincident_i, info.coincident_j
            if order is not None:
                i, j = sorted((int(order[i]), int(order[j])))
            raise RuntimeError(f"Coincident atoms: {i}:: == {j}::")
        if info.status & _lib.ST_NEAR_OVERFLOW:
            raise RuntimeError("too many nearby low probes for one probe (limit 512)")
        self._n = len(rad)
        self._n0 = n0
        self._order = order
        self._sc_done = [False]
        self.run._state = (self._lease, (xyz, rad, dens, mol), len(rad), n0, self._sc_done, order)
        self.run.radmax = np.float64(rad.max())
        r = self.run.results
        r.dots.convex += int(info.convex)
        r.dots.toroidal += int(info.toroidal)
        r.dots.concave += int(info.concave)
        for m in (0, 1):
            # assign_attention_numbers' counters (_core.py:1160-1193)
            if not all_atoms:
                r.surface[m].nBlockedAtoms += int(info.n_blocked[m])
            r.surface[m].nBuriedAtoms += int(info.n_attended[m])
        self.run.surfaces_generated = True
        self.run.surfaces_generated_all_atoms = all_atoms

    def generate_molecular_surfaces(self):
        self._ensure_surfaces_generated(all_atoms=False)

    # -- readouts ---------------------------------------------------------------
    def CalcLoaded(self):
        self.run.results.valid = 0
        self._ensure_surfaces_generated(all_atoms=False)
        return self.calc_contact_molecular_surface(target_side=True)

    def CalcLoadedMaxPossibleCMS(self):
        self.run.results.valid = 0
        self._ensure_surfaces_generated(all_atoms=True)
        return self.calc_max_possible_contact_molecular_surface(target_side=True)

    def calc_contact_molecular_surface(self, target_side=True):
        """(total, per-atom array of the query molecule); target_side=True: query = target."""
        if self._cms is None:
            self._cms = self._context().contact_ms()
        per_atom, totals = self._cms
        n0 = self._n0
        if target_side:
            return float(totals[0, 1]), per_atom[n0:self._n].copy()
        return float(totals[0, 0]), per_atom[:n0].copy()

    def calc_contact_molecular_surface_gradient(self, target_side=True):
        """
        d(CMS)/d(xyz) of every loaded atom (N x 3, rows in AddMolecule order)
        for the target-side (or binder-side)
        CMS, with the generated dot topology held fixed.  The reference has
        no gradient; this is the FP64 adjoint of calc_contact_molecular_surface.
        """
        self._ensure_surfaces_generated(all_atoms=False)
        if self._cms is None:
            self.calc_contact_molecular_surface(target_side)
        g = self._context().contact_ms_backward(target_side=target_side)
        if self._order is None:
            return g
        out = np.empty_like(g)
        out[self._order] = g
        return out

    def calc_max_possible_contact_molecular_surface(self, target_side=True):
        if self._max is None:
            self._max = self._context().max_contact_ms()
        per_atom, totals = self._max
        return float(totals[0]), per_atom[:self._n0].copy()

    def CalcLoadedSC(self):
        self.run.results.valid = 0
        self._ensure_surfaces_generated(all_atoms=False)
        if self._sc is None:
            self._sc = self._context().shape_complementarity()
            self._sc_done[0] = True
            self.run._host.pop("trimmed_dots", None)
        sc, sides = self._sc
        res = self.run.results
        for m in (0, 1):
            s = res.surface[m]
            v = sides[0, m]
            s.d_mean, s.d_median, s.s_mean, s.s_median, s.trimmedArea = (float(v[0]), float(v[1]), float(v[2]),
                                                                        float(v[3]), float(v[4]))
            s.nTrimmedDots = int(v[5])
            s.nAllDots = int(v[6])
        s0, s1, s2 = res.surface
        s2.d_mean = (s0.d_mean + s1.d_mean) / 2
        s2.d_median = (s0.d_median + s1.d_median) / 2
        s2.s_mean = (s0.s_mean + s1.s_mean) / 2
        s2.s_median = (s0.s_median + s1.s_median) / 2
        s2.nAllDots = s0.nAllDots + s1.nAllDots
        s2.nTrimmedDots = s0.nTrimmedDots + s1.nTrimmedDots
        s2.trimmedArea = s0.trimmedArea + s1.trimmedArea
        res.sc = s2.s_median
        res.distance = s2.d_median
        res.area = s2.trimmedArea
        res.valid = 1
        return res.sc, res.area, res.distance


MolecularSurfaceCalculatorGPU = MolecularSurfaceCalculator
