"""
GPU parity against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's CPU calculator).

Checks the contract of the reference's parity test (test/test_gpu_parity.py):
identical dot / probe / toroid / neighbour counts, flags and ownership, and
floating-point values within 1e-12 (scaled) of the reference.
"""

import numpy as np
import pytest

from parity import ALL_CASES, FULL_CASES, close, exact, inputs, load_case

pytestmark = pytest.mark.gpu


def _calc():
    from cms_cuda import MolecularSurfaceCalculator
    return MolecularSurfaceCalculator()


@pytest.fixture(scope="module")
def runs():
    out = {}
    for name in ALL_CASES:
        case = load_case(name)
        bx, br, tx, tr = inputs(case)
        calc = _calc()
        calc.add_binder_and_target(bx, br, tx, tr)
        cms, pa = calc.CalcLoaded()
        bcms, pb = calc.calc_contact_molecular_surface(target_side=False)
        sc = calc.CalcLoadedSC()
        mcalc = _calc()
        mcalc.AddMolecule(0, tx, tr)
        mx, mpa = mcalc.CalcLoadedMaxPossibleCMS()
        out[name] = dict(case=case, calc=calc, cms=cms, pa=pa, bcms=bcms, pb=pb, sc=sc, mcalc=mcalc, mx=mx, mpa=mpa)
    return out


@pytest.mark.parametrize("name", ALL_CASES)
def test_cms_values(runs, name):
    R = runs[name]
    c = R["case"]
    assert type(R["cms"]) is float and type(R["bcms"]) is float and type(R["mx"]) is float
    assert isinstance(R["pa"], np.ndarray) and len(R["pa"]) == len(c["tx"]) and len(R["pb"]) == len(c["bx"])
    close("cms target", R["cms"], c["cms"])
    close("cms binder", R["bcms"], c["cms_binder"])
    close("per-atom target", R["pa"], c["per_atom_target"])
    close("per-atom binder", R["pb"], c["per_atom_binder"])
    close("max cms", R["mx"], c["max_cms"])
    close("max per-atom", R["mpa"], c["per_atom_max"])


@pytest.mark.parametrize("name", ALL_CASES)
def test_sc_values(runs, name):
    R = runs[name]
    c = R["case"]
    close("sc", R["sc"][0], c["sc"])
    close("sc area", R["sc"][1], c["sc_area"])
    close("sc distance", R["sc"][2], c["sc_distance"])
    res = R["calc"].run.results
    for m in range(3):
        s = res.surface[m]
        got = [s.d_mean, s.d_median, s.s_mean, s.s_median, s.trimmedArea, s.nTrimmedDots, s.nAllDots,
               s.nBuriedAtoms, s.nBlockedAtoms]
        close(f"surface[{m}]", got, c["surface"][m])


@pytest.mark.parametrize("name", ALL_CASES)
def test_counts_and_flags(runs, name):
    R = runs[name]
    c = R["case"]
    calc = R["calc"]
    r = calc.run
    exact("dot type counts", [r.results.dots.convex, r.results.dots.toroidal, r.results.dots.concave], c["counts"])
    exact("probes", len(r.probes), int(c["n_probes"]))
    exact("toroid queue", len(r.toroid_queue), int(c["n_toroid"]))
    exact("atten", r.atoms.atten, c["atten"])
    exact("access", r.atoms.access, c["access"])
    exact("n neighbours", r.neighbor_array.nneighbors, c["nn"])
    exact("n buried partners", r.buried_array.nneighbors, c["nbur"])
    exact("radmax", float(r.radmax), float(c["radmax"]))
    nb = len(c["bx"])
    for m in (0, 1):
        d = r.dots[m]
        off = 0 if m == 0 else nb
        nat = nb if m == 0 else len(c["tx"])
        exact(f"dots[{m}] count", len(d), int(c[f"n_dots{m}"]))
        exact(f"dots[{m}] per-atom count", np.bincount(d.atom_idx - off, minlength=nat), c[f"dot_count_atom{m}"])
        exact(f"dots[{m}] per-atom buried", np.bincount(d.atom_idx - off, weights=d.buried.astype(float),
                                                        minlength=nat).astype(np.int64), c[f"dot_buried_atom{m}"])
        exact(f"dots[{m}] buried", int(d.buried.sum()), int(c[f"n_buried{m}"]))
        for t in (1, 2, 3):
            exact(f"dots[{m}] type {t}", int((d.type_ == t).sum()), int(c[f"n_type{t}_{m}"]))
        exact(f"trimmed[{m}] count", len(r.trimmed_dots[m]), int(c[f"n_trimmed{m}"]))
        if f"dots{m}_atom" in c:
            # every dot's owner, burial flag and type (all fixtures keep them; the large plain complex too)
            exact(f"dots[{m}].atom_idx", d.atom_idx, c[f"dots{m}_atom"])
            exact(f"dots[{m}].buried", d.buried, c[f"dots{m}_buried"])
            exact(f"dots[{m}].type_", d.type_, c[f"dots{m}_type"])
    mr = R["mcalc"].run
    exact("max-cms dot counts", [mr.results.dots.convex, mr.results.dots.toroidal, mr.results.dots.concave],
          c["max_counts"])
    exact("max-cms access", mr.atoms.access, c["max_access"])
    exact("max-cms per-atom dots", np.bincount(mr.dots[0].atom_idx, minlength=len(c["tx"])), c["max_dot_count_atom"])


@pytest.mark.parametrize("name", FULL_CASES)
def test_full_run_state(runs, name):
    R = runs[name]
    c = R["case"]
    r = R["calc"].run
    for m in (0, 1):
        d = r.dots[m]
        exact(f"dots[{m}].buried", d.buried, c[f"dots{m}_buried"])
        exact(f"dots[{m}].type_", d.type_, c[f"dots{m}_type"])
        exact(f"dots[{m}].atom_idx", d.atom_idx, c[f"dots{m}_atom"])
        close(f"dots[{m}].coor_xyz", d.coor_xyz, c[f"dots{m}_coor"])
        close(f"dots[{m}].outnml_xyz", d.outnml_xyz, c[f"dots{m}_nml"])
        close(f"dots[{m}].area", d.area, c[f"dots{m}_area"])
        t = r.trimmed_dots[m]
        exact(f"trimmed[{m}].atom_idx", t.atom_idx, c[f"trim{m}_atom"])
        close(f"trimmed[{m}].coor_xyz", t.coor_xyz, c[f"trim{m}_coor"])
    p = r.probes
    exact("probe atoms", np.stack([p.atom_idx_0, p.atom_idx_1, p.atom_idx_2], 1), c["probe_atoms"])
    close("probe height", p.height, c["probe_height"])
    close("probe point", p.point_xyz, c["probe_point"])
    close("probe alt", p.alt_xyz, c["probe_alt"])
    tq = r.toroid_queue
    exact("toroid atoms", np.array([(t[0], t[1]) for t in tq], dtype=np.int32).reshape(-1, 2), c["tor_atoms"])
    exact("toroid between", np.array([t[5] for t in tq], dtype=bool), c["tor_between"])
    close("toroid uij", np.array([t[2] for t in tq]).reshape(-1, 3), c["tor_uij"])
    close("toroid tij", np.array([t[3] for t in tq]).reshape(-1, 3), c["tor_tij"])
    close("toroid rij", np.array([t[4] for t in tq]), c["tor_rij"])
    exact("neighbour rows", r.neighbor_array.natom, c["nb_natom"])
    exact("buried rows", r.buried_array.natom, c["bu_natom"])
    md = R["mcalc"].run.dots[0]
    close("max-cms dot areas", md.area, c["max_dots0_area"])
    exact("max-cms dot atoms", md.atom_idx, c["max_dots0_atom"])


def test_pickle_goldens(runs):
    """The reference's own regression pickles (test/golden.pkl, test/sc_golden.pkl)."""
    R = runs["golden_pkl"]
    c = R["case"]
    close("golden.pkl cms", R["cms"], float(c["pkl_cms"]))
    close("sc_golden.pkl sc", R["sc"][0], float(c["pkl_sc"]))
    close("sc_golden.pkl area", R["sc"][1], float(c["pkl_sc_area"]))
    close("sc_golden.pkl distance", R["sc"][2], float(c["pkl_sc_distance"]))
    r = R["calc"].run
    exact("golden.pkl dots", [len(r.dots[0]), len(r.dots[1])], c["pkl_dots"])
    exact("sc_golden.pkl trimmed", [len(r.trimmed_dots[0]), len(r.trimmed_dots[1])], c["pkl_trimmed"])


def test_shared_cache_and_mode_mismatch(runs):
    """CalcLoaded and CalcLoadedSC share one surface; max-CMS on it raises (_core.py:882-893)."""
    c = runs["golden_pkl"]["case"]
    calc = _calc()
    calc.add_binder_and_target(*inputs(c))
    sc1 = calc.CalcLoadedSC()
    cms1 = calc.CalcLoaded()[0]
    close("cms after sc", cms1, c["cms"])
    close("sc before cms", sc1[0], c["sc"])
    with pytest.raises(RuntimeError):
        calc.CalcLoadedMaxPossibleCMS()


def test_deterministic(runs):
    """Two GPU runs are bit-identical."""
    c = runs["synth_small_s7"]["case"]
    outs = []
    for _ in range(2):
        calc = _calc()
        calc.add_binder_and_target(*inputs(c))
        cms, pa = calc.CalcLoaded()
        sc = calc.CalcLoadedSC()
        outs.append((cms, pa, sc, calc.run.dots[1].coor_xyz.copy()))
    assert outs[0][0] == outs[1][0]
    exact("per-atom", outs[0][1], outs[1][1])
    exact("sc", outs[0][2], outs[1][2])
    exact("dots", outs[0][3], outs[1][3])


def test_public_api(runs):
    from cms_cuda import (calculate_contact_ms, calculate_maximum_possible_contact_ms,
                          calculate_shape_complementarity)
    c = runs["golden_pkl"]["case"]
    bx, br, tx, tr = inputs(c)
    cms, pa, calc = calculate_contact_ms(bx, br, tx, tr)
    close("api cms", cms, c["cms"])
    sc, area, dist, _ = calculate_shape_complementarity(bx, br, tx, tr, device="cuda")
    close("api sc", sc, c["sc"])
    mx, mpa, _ = calculate_maximum_possible_contact_ms(tx, tr, device="gpu")
    close("api max", mx, c["max_cms"])
    with pytest.raises(ValueError):
        calculate_contact_ms(bx, br, tx, tr, device="cpu")


def test_graph_capacity_overflow_is_detected_and_recovered():
    """
    A graph captured on a batch with a smaller surface (the first complex's
    binder 100 A away) replayed on the same shape with both complexes in
    contact exceeds its capacities: the run is
    flagged (every later kernel stops at entry), graph_check reports it, and
    run_graph re-sizes and returns the exact results.
    """
    from cms_cuda import _lib
    names = ("golden_pkl", "synth_small_s7")
    xyz, rad, off, nb = [], [], [0], []
    for n in names:
        bx, br, tx, tr = inputs(load_case(n))
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    X, R = np.concatenate(xyz), np.concatenate(rad)
    off, nb = np.array(off), np.array(nb)
    far = X.copy()
    far[off[0]:off[0] + nb[0], 0] += 100.0
    ctx = _lib.Context(0)
    ctx.load_batch(off, nb, far, R)
    ctx.run_graph()
    ctx.load_batch(off, nb, X, R)
    ctx.graph_launch()
    with pytest.raises(_lib.CmsError):
        ctx.graph_check()
    ctx.run_graph()
    _, tot = ctx.contact_ms(per_atom=False)
    sc, _ = ctx.shape_complementarity()
    ref = _lib.Context(0)
    ref.load_batch(off, nb, X, R)
    ref.generate(all_atoms=False)
    _, rtot = ref.contact_ms(per_atom=False)
    rsc, _ = ref.shape_complementarity()
    exact("totals after recovery", tot, rtot)
    exact("sc after recovery", sc, rsc)


def test_probe_stash_and_recompute_agree():
    """
    The triple count pass stashes its probes when they fit the capacity it
    ran with, and a scatter fills the probe arrays; otherwise (the first run
    of a fresh context) the emit pass recomputes them.  Likewise the convex
    count pass keeps its accepted candidates, the concave count pass makes
    its dots, the toroidal count pass keeps its torus points with arc dots
    and the neighbour count pass its rows for the emit passes.  Both ways
    give the same neighbour lists, probes, dots, access flags and results.
    """
    from cms_cuda import _lib
    names = ("golden_pkl", "synth_small_s7", "synth_zero_radii")
    xyz, rad, off, nb = [], [], [0], []
    for n in names:
        bx, br, tx, tr = inputs(load_case(n))
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    X, R = np.concatenate(xyz), np.concatenate(rad)
    off, nb = np.array(off), np.array(nb)
    ctx = _lib.Context(0)
    ctx.load_batch(off, nb, X, R)

    def snapshot():
        out = []
        for c in range(len(names)):
            i = ctx.info(c)
            n = int(off[c + 1] - off[c])
            out.append(ctx.export_probes(c, i) + ctx.export_atoms(c, n) + ctx.export_dots(c, 0, i)
                       + ctx.export_dots(c, 1, i) + ctx.export_neighbors(c, n, i))
        return out, ctx.contact_ms(per_atom=True)

    ctx.generate(all_atoms=False)          # capacities sized by this run: recomputed
    first, cms1 = snapshot()
    ctx.generate(all_atoms=False)          # capacities fit: stashed and scattered
    second, cms2 = snapshot()
    assert sum(len(p[0]) for p in first) > 0
    for a, b in zip(first, second):
        for x, y in zip(a, b):
            exact("probe arrays", x, y)
    exact("per-atom cms", cms1[0], cms2[0])
    for c, n in enumerate(names):
        case = load_case(n)
        if "probe_point" in case:
            close("probes vs reference", second[c][4], case["probe_point"])
