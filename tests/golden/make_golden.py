"""
Generate the golden fixtures in this directory by running the reference
implementation (ullahsamee/cms-cuda, CPU calculator cms-cuda/_core.py).

Needs a checkout of the reference, named by the environment variable
CMS_REFERENCE_DIR (it is not available where the GPU tests run, which is why
the outputs are committed).  The reference's
own regression pickles (test/golden.pkl, test/sc_golden.pkl) are read with a
restricted unpickler that admits only the three globals they contain.

Each fixture ``<case>.npz`` holds the inputs (binder/target xyz and radii),
the reference's scalar outputs, per-atom arrays, and for small cases the full
run state (dots, probes, toroid queue, neighbour lists, trimmed dots).  The
large plain complex also keeps every dot's owner atom, burial flag and type.

``synth_small_s7_order.npz`` holds the reference's run state when the
molecules of ``synth_small_s7`` are added target first, and interleaved.

``batched_4096_sample.npz`` holds eight complexes of the batched workload
(4096 complexes, seed 2): the smallest, the largest, the 10th / 50th / 90th
size percentiles, the complex with the largest binder and the smallest and
largest complexes (among the others) whose binder is a ligand-like HETATM
C*/N*/O* cluster.
Keys are prefixed ``k<slot>_``; every dot's owner, burial flag and type are
kept.

Usage:  CMS_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py [case ...]
"""

import importlib.util
import io
import os
import pickle
import sys

import numpy as np

REF = os.environ.get("CMS_REFERENCE_DIR", "")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cms-cuda_b200"))


def load_reference_core():
    spec = importlib.util.spec_from_file_location("ref_core", os.path.join(REF, "cms-cuda", "_core.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Snapshot:
    """Stand-in for the pickles' __main__.TestCalculatorRun (plain attribute bag)."""


def read_golden_pickle(path):
    import numpy._core.multiarray as ma

    allowed = {("__main__", "TestCalculatorRun"): _Snapshot,
               ("numpy._core.multiarray", "scalar"): ma.scalar,
               ("numpy", "dtype"): np.dtype}

    class Restricted(pickle.Unpickler):
        def find_class(self, module, name):
            if (module, name) in allowed:
                return allowed[(module, name)]
            raise pickle.UnpicklingError(f"global {module}.{name} is not allowed")

    with open(path, "rb") as fh:
        return Restricted(io.BytesIO(fh.read())).load()


def pickle_inputs(g):
    mol = np.array([a["molecule"] for a in g.atoms])
    xyz = np.array([[a["x"], a["y"], a["z"]] for a in g.atoms])
    rad = np.array([a["radius"] for a in g.atoms])
    return xyz[mol == 0], rad[mol == 0], xyz[mol == 1], rad[mol == 1]


def assert_no_distance_ties(bx, tx):
    """
    The reference orders each neighbour row with np.argsort (unstable) on d2
    alone (_core.py:1331); an exact d2 tie inside a row makes its order
    implementation-defined, so fixture inputs must not contain one.
    """
    for xyz in (bx, tx):
        d = xyz[:, None, :] - xyz[None, :, :]
        d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
        np.fill_diagonal(d2, np.inf)
        d2 = np.where(d2 < 64.0, d2, np.inf)
        s = np.sort(d2, axis=1)
        ties = (s[:, 1:] == s[:, :-1]) & np.isfinite(s[:, 1:])
        assert not ties.any(), "exact neighbour-distance tie in fixture input"


def run_reference(core, bx, br, tx, tr, full, max_cms=True, dots=False):
    assert_no_distance_ties(bx, tx)
    calc = core.MolecularSurfaceCalculator()
    calc.add_binder_and_target(bx, br, tx, tr)
    cms, pa = calc.CalcLoaded()
    bcms, pb = calc.calc_contact_molecular_surface(target_side=False)
    sc, sc_area, sc_dist = calc.CalcLoadedSC()
    r = calc.run
    out = dict(bx=bx, br=br, tx=tx, tr=tr, cms=cms, cms_binder=bcms, sc=sc, sc_area=sc_area, sc_distance=sc_dist,
               per_atom_target=pa, per_atom_binder=pb,
               counts=np.array([r.results.dots.convex, r.results.dots.toroidal, r.results.dots.concave]),
               n_probes=len(r.probes), n_toroid=len(r.toroid_queue), radmax=float(r.radmax),
               atten=r.atoms.atten.copy(), access=r.atoms.access.copy(),
               nn=r.neighbor_array.nneighbors.copy(), nbur=r.buried_array.nneighbors.copy())
    if max_cms:
        mx, mpa, mcalc = core.calculate_maximum_possible_contact_ms(tx, tr)
        out.update(max_cms=mx, per_atom_max=mpa, max_access=mcalc.run.atoms.access.copy(),
                   max_counts=np.array([mcalc.run.results.dots.convex, mcalc.run.results.dots.toroidal,
                                        mcalc.run.results.dots.concave]))
    surf = np.array([[getattr(s, k) for k in ("d_mean", "d_median", "s_mean", "s_median", "trimmedArea",
                                                "nTrimmedDots", "nAllDots", "nBuriedAtoms", "nBlockedAtoms")]
                     for s in r.results.surface], dtype=np.float64)
    out["surface"] = surf
    n = len(r.atoms)
    for m in (0, 1):
        d = r.dots[m]
        nat = len(bx) if m == 0 else len(tx)
        off = 0 if m == 0 else len(bx)
        out[f"dot_count_atom{m}"] = np.bincount(d.atom_idx - off, minlength=nat)
        out[f"dot_buried_atom{m}"] = np.bincount(d.atom_idx - off, weights=d.buried.astype(float),
                                                 minlength=nat).astype(np.int64)
        out[f"n_dots{m}"] = len(d)
        out[f"n_buried{m}"] = int(d.buried.sum())
        out[f"n_trimmed{m}"] = len(r.trimmed_dots[m])
        for t in (1, 2, 3):
            out[f"n_type{t}_{m}"] = int((d.type_ == t).sum())
    if max_cms:
        md = mcalc.run.dots[0]
        out["max_dot_count_atom"] = np.bincount(md.atom_idx, minlength=len(tx))
    if dots and not full:
        for m in (0, 1):
            d = r.dots[m]
            out[f"dots{m}_buried"] = d.buried
            out[f"dots{m}_type"] = d.type_
            out[f"dots{m}_atom"] = d.atom_idx
    if full:
        for m in (0, 1):
            d = r.dots[m]
            out[f"dots{m}_coor"] = d.coor_xyz
            out[f"dots{m}_nml"] = d.outnml_xyz
            out[f"dots{m}_area"] = d.area
            out[f"dots{m}_buried"] = d.buried
            out[f"dots{m}_type"] = d.type_
            out[f"dots{m}_atom"] = d.atom_idx
            td = r.trimmed_dots[m]
            out[f"trim{m}_coor"] = td.coor_xyz
            out[f"trim{m}_atom"] = td.atom_idx
        p = r.probes
        out["probe_atoms"] = np.stack([p.atom_idx_0, p.atom_idx_1, p.atom_idx_2], 1)
        out["probe_height"], out["probe_point"], out["probe_alt"] = p.height, p.point_xyz, p.alt_xyz
        tq = r.toroid_queue
        out["tor_atoms"] = np.array([(t[0], t[1]) for t in tq], dtype=np.int32).reshape(-1, 2)
        out["tor_uij"] = np.array([t[2] for t in tq]).reshape(-1, 3)
        out["tor_tij"] = np.array([t[3] for t in tq]).reshape(-1, 3)
        out["tor_rij"] = np.array([t[4] for t in tq])
        out["tor_between"] = np.array([t[5] for t in tq], dtype=bool)
        na = r.neighbor_array
        out["nb_natom"] = na.natom
        out["bu_natom"] = r.buried_array.natom
        out["max_dots0_area"] = md.area
        out["max_dots0_atom"] = md.atom_idx
    return out


BATCH_B, BATCH_SEED = 4096, 2


def batched_sample_indices(batch):
    """Eight complexes stratified over the batched workload (see the module docstring)."""
    sizes = np.diff(batch.atom_off)
    order = np.argsort(sizes, kind="stable")
    pick = [int(order[0]), int(order[-1])]
    pick += [int(order[int(q * (len(order) - 1))]) for q in (0.1, 0.5, 0.9)]
    pick.append(int(np.argmax(batch.n_binder)))
    lig = np.nonzero(batch.ligand)[0]
    lig = [int(c) for c in lig[np.argsort(sizes[lig], kind="stable")] if int(c) not in pick]
    pick += [lig[0], lig[-1]]
    assert len(set(pick)) == len(pick) and sum(bool(batch.ligand[c]) for c in pick) >= 2
    return pick


def make_batched_sample(core):
    from cms_cuda import synth
    batch = synth.config_batched(BATCH_B, BATCH_SEED)
    pick = batched_sample_indices(batch)
    out = dict(batch_index=np.array(pick, np.int64), ligand=batch.ligand[pick])
    for k, c in enumerate(pick):
        r = run_reference(core, *batch.complex(c), full=False, max_cms=False, dots=True)
        for key, v in r.items():
            out[f"k{k}_{key}"] = v
        print(f"  batched complex {c} (slot {k}, ligand {bool(batch.ligand[c])}): atoms "
              f"{len(r['br'])}+{len(r['tr'])} dots={r['n_dots0']}+{r['n_dots1']} cms={r['cms']:.10g}", flush=True)
    path = os.path.join(HERE, "batched_4096_sample.npz")
    np.savez_compressed(path, **out)
    print(f"batched_4096_sample -> {os.path.getsize(path) / 1e6:.2f} MB", flush=True)


def add_dot_ownership(core, name):
    """Add every dot's owner, burial flag and type to an existing fixture (CMS surface only)."""
    path = os.path.join(HERE, name + ".npz")
    with np.load(path) as z:
        case = {k: z[k] for k in z.files}
    assert_no_distance_ties(case["bx"], case["tx"])
    calc = core.MolecularSurfaceCalculator()
    calc.add_binder_and_target(case["bx"], case["br"], case["tx"], case["tr"])
    cms, _ = calc.CalcLoaded()
    assert cms == case["cms"]
    for m in (0, 1):
        d = calc.run.dots[m]
        assert len(d) == case[f"n_dots{m}"]
        case[f"dots{m}_buried"] = d.buried
        case[f"dots{m}_type"] = d.type_
        case[f"dots{m}_atom"] = d.atom_idx
    np.savez_compressed(path, **case)
    print(f"{name}: per-dot owner / burial / type added -> {os.path.getsize(path) / 1e6:.2f} MB", flush=True)


ORDER_CASES = {
    # AddMolecule calls as (molecule, binder or target, first atom, end atom) over synth_small_s7's inputs
    "target_first": ((1, "t", 0, None), (0, "b", 0, None)),
    "interleaved": ((0, "b", 0, 70), (1, "t", 0, 150), (0, "b", 70, None), (1, "t", 150, None)),
}


def make_order_cases(core):
    """
    The reference with molecules added out of binder-first order: its surface,
    SC and run state, and its binder-side readout.  Its target-side readout
    indexes per-atom bins by natom minus the molecule-0 atom count
    (_core.py:990-995), which is negative for target atoms numbered before
    binder atoms, so np.bincount raises there; that is recorded, not stored.
    """
    from cms_cuda import synth  # noqa: F401  (keeps the import path of the other cases)
    base = dict(np.load(os.path.join(HERE, "synth_small_s7.npz")))
    src = {"b": (base["bx"], base["br"]), "t": (base["tx"], base["tr"])}
    out = {}
    for name, calls in ORDER_CASES.items():
        calc = core.MolecularSurfaceCalculator()
        for mol, side, a, b in calls:
            x, r = src[side]
            calc.AddMolecule(mol, x[a:b], r[a:b])
        try:
            calc.CalcLoaded()
            out[f"{name}_target_raises"] = False
        except ValueError:
            out[f"{name}_target_raises"] = True
        bcms, pb = calc.calc_contact_molecular_surface(target_side=False)
        sc = calc.CalcLoadedSC()
        r = calc.run
        out[f"{name}_cms_binder"] = bcms
        out[f"{name}_per_atom_binder"] = pb
        out[f"{name}_sc"] = np.array(sc)
        out[f"{name}_molecule"] = r.atoms.molecule.copy()
        out[f"{name}_atten"] = r.atoms.atten.copy()
        out[f"{name}_access"] = r.atoms.access.copy()
        for m in (0, 1):
            d = r.dots[m]
            # positions and areas are those of the binder-first run (kept in synth_small_s7.npz)
            assert np.array_equal(d.coor_xyz, base[f"dots{m}_coor"]) and np.array_equal(d.area, base[f"dots{m}_area"])
            out[f"{name}_dots{m}_buried"] = d.buried
            out[f"{name}_dots{m}_atom"] = d.atom_idx
            out[f"{name}_trim{m}_atom"] = r.trimmed_dots[m].atom_idx
        p = r.probes
        out[f"{name}_probe_atoms"] = np.stack([p.atom_idx_0, p.atom_idx_1, p.atom_idx_2], 1)
        out[f"{name}_probe_point"] = p.point_xyz
        tq = r.toroid_queue
        out[f"{name}_tor_atoms"] = np.array([(t[0], t[1]) for t in tq], dtype=np.int32).reshape(-1, 2)
        out[f"{name}_tor_tij"] = np.array([t[3] for t in tq]).reshape(-1, 3)
        out[f"{name}_nb_natom"] = r.neighbor_array.natom
        out[f"{name}_nb_count"] = r.neighbor_array.nneighbors
        out[f"{name}_bu_natom"] = r.buried_array.natom
        print(f"  {name}: target side raises {out[f'{name}_target_raises']}, binder cms {bcms:.10g}, "
              f"sc {sc[0]:.10g}", flush=True)
    path = os.path.join(HERE, "synth_small_s7_order.npz")
    np.savez_compressed(path, **out)
    print(f"synth_small_s7_order -> {os.path.getsize(path) / 1e6:.2f} MB", flush=True)


def main():
    if not os.path.isdir(os.path.join(REF, "cms-cuda")):
        sys.exit("set CMS_REFERENCE_DIR to a checkout of the reference (the directory holding cms-cuda/)")
    core = load_reference_core()
    only = set(sys.argv[1:])
    if "batched_4096_sample" in only:
        make_batched_sample(core)
        only.discard("batched_4096_sample")
        if not only:
            return
    if "synth_small_s7_order" in only:
        make_order_cases(core)
        only.discard("synth_small_s7_order")
        if not only:
            return
    if "dot_ownership_8000_1800" in only:
        add_dot_ownership(core, "synth_plain_8000_1800")
        only.discard("dot_ownership_8000_1800")
        if not only:
            return
    cases = []
    g = read_golden_pickle(os.path.join(REF, "test", "golden.pkl"))
    gs = read_golden_pickle(os.path.join(REF, "test", "sc_golden.pkl"))
    cases.append(("golden_pkl", pickle_inputs(g), True,
                  dict(pkl_cms=g.cms, pkl_sc=gs.sc, pkl_sc_area=gs.results["area"],
                       pkl_sc_distance=gs.results["distance"],
                       pkl_dots=np.array([len(g.dots[0]), len(g.dots[1])]),
                       pkl_counts=np.array([g.results["dots_convex"], g.results["dots_toroidal"],
                                            g.results["dots_concave"]]),
                       pkl_trimmed=np.array([len(gs.trimmed_dots[0]), len(gs.trimmed_dots[1])]))))
    from cms_cuda.structure import load_complex
    cases.append(("sc_example_pdb", load_complex(os.path.join(REF, "test", "sc_example.pdb")), False, {}))
    cases.append(("smallmol_7jkv_pdb", load_complex(os.path.join(REF, "examples", "7jkv-smallmol.pdb")), False, {}))
    from cms_cuda import synth
    cases.append(("synth_small_s7", synth.make_complex(300, 120, 7), True, {}))
    bx, br, tx, tr = synth.make_complex(400, 150, 11)
    br = br.copy(); tr = tr.copy()
    br[::11] = 0.0                 # radius-0 atoms are kept (test_gpu_parity.py:102-107)
    tr[5::11] = 0.0
    cases.append(("synth_zero_radii", (bx, br, tx, tr), True, {}))
    cases.append(("synth_plain_1200_450", synth.config_plain_small(0), False, {}))
    cases.append(("synth_plain_8000_1800", synth.config_plain_large(0), False, {}))
    for name, inputs, full, extra in cases:
        if only and name not in only:
            continue
        out = run_reference(core, *inputs, full=full)
        out.update(extra)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: atoms {len(inputs[0])}+{len(inputs[2])} cms={out['cms']:.10g} sc={out['sc']:.10g} "
              f"dots={out['n_dots0']}+{out['n_dots1']} -> {os.path.getsize(path) / 1e6:.2f} MB", flush=True)


if __name__ == "__main__":
    main()
