"""
The standalone nearest-dot search (cms_nearest_dots) against SciPy's
cdist(ref, query, 'sqeuclidean').min(axis=0) / .argmin(axis=0), the CPU
computation the reference's min_sqdist primitive replaces
(cms-cuda/_gpu_kernels.py:508-566): bit-identical minima and first-index
argmins, exact ties included.
"""

import numpy as np
import pytest
from scipy.spatial.distance import cdist

from parity import exact, load_case

pytestmark = pytest.mark.gpu


def _ctx():
    from cms_cuda import _lib
    return _lib.Context(0)


def test_random_points_with_ties():
    rng = np.random.default_rng(0)
    q = rng.uniform(-30, 30, (3000, 3))
    r = rng.uniform(-30, 30, (7000, 3))
    r[4100] = r[50]            # duplicate reference: the first index must win
    q[7] = r[50]               # a query sitting on it (distance 0)
    q[8] = (r[10] + r[20]) / 2
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))
    assert idx[7] == 50 and d2[7] == 0.0


def test_golden_buried_dots():
    """Buried target dots against buried binder dots of the reference's golden complex."""
    c = load_case("golden_pkl")
    q = c["dots1_coor"][c["dots1_buried"] == 1]
    r = c["dots0_coor"][c["dots0_buried"] == 1]
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))


def test_far_offset_coordinates():
    """Large absolute coordinates (FP32 staging relative to the box centre)."""
    rng = np.random.default_rng(1)
    base = np.array([5000.0, -3000.0, 12000.0])
    q = base + rng.normal(0, 10, (500, 3))
    r = base + rng.normal(0, 10, (900, 3))
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_search_shapes_give_identical_results(variant):
    """Every tunable search shape returns the default shape's CMS, SC and gradient bit for bit."""
    from cms_cuda import _lib
    from parity import inputs, load_case
    cases = [load_case(n) for n in ("golden_pkl", "synth_small_s7", "sc_example_pdb")]
    xyz, rad, off, nb = [], [], [0], []
    for c in cases:
        bx, br, tx, tr = inputs(c)
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    X, R = np.concatenate(xyz), np.concatenate(rad)
    out = []
    for v in (0, variant):
        ctx = _lib.Context(0)
        ctx.set_nn_variants([v, v, v])
        ctx.load_batch(np.array(off), np.array(nb), X, R)
        ctx.generate(all_atoms=False)
        pa, tot = ctx.contact_ms(per_atom=True)
        sc, sides = ctx.shape_complementarity()
        g = ctx.contact_ms_backward(True)
        out.append((pa, tot, sc, sides, g))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b, equal_nan=True)


def test_autotuner_picks_shapes():
    from cms_cuda import _lib
    from parity import inputs, load_case
    bx, br, tx, tr = inputs(load_case("synth_plain_1200_450"))
    ctx = _lib.Context(0)
    ctx.load_batch(np.array([0, len(br) + len(tr)]), np.array([len(br)]), np.concatenate([bx, tx]),
                   np.concatenate([br, tr]))
    ctx.run_graph()
    v, ms = ctx.nn_variants()
    assert all(0 <= x < 4 for x in v)
    assert np.isfinite(ms).all() and (ms > 0).all()
    for k in range(3):
        assert ms[k, v[k]] == ms[k].min()


@pytest.mark.parametrize("graph", [False, True], ids=["staged", "graph"])
def test_surface_shapes_give_identical_surfaces(graph):
    """Every toroidal / concave kernel shape the autotuner may pick generates the same dots, bit for bit."""
    from cms_cuda import _lib
    from parity import inputs, load_case
    names = ("golden_pkl", "synth_small_s7", "synth_zero_radii", "smallmol_7jkv_pdb")
    xyz, rad, off, nb = [], [], [0], []
    for n in names:
        bx, br, tx, tr = inputs(load_case(n))
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    X, R = np.concatenate(xyz), np.concatenate(rad)
    out = []
    for v in ([0, 0, 0, 0, 0], [1, 1, 1, 1, 1], [2, 2, 2, 2, 2], [1, 0, 2, 1, 1]):
        ctx = _lib.Context(0)
        ctx.set_surface_variants(v)
        ctx.load_batch(np.array(off), np.array(nb), X, R)
        if graph:
            ctx.run_graph()
            ctx.graph_launch()             # a replay with the stashes of the captured run
        else:
            ctx.generate(all_atoms=False)
        dots = []
        for c in range(len(names)):
            i = ctx.info(c)
            dots += [ctx.export_dots(c, m, i) for m in (0, 1)]
        pa, tot = ctx.contact_ms(per_atom=True)
        assert ctx.surface_variants()[0] == v
        out.append((dots, pa, tot))
    for other in out[1:]:
        for a, b in zip(out[0][0], other[0]):
            for x, y in zip(a, b):
                assert np.array_equal(x, y, equal_nan=True)
        assert np.array_equal(out[0][1], other[1]) and np.array_equal(out[0][2], other[2])


def test_autotuner_picks_surface_shapes():
    from cms_cuda import _lib
    from parity import inputs, load_case
    bx, br, tx, tr = inputs(load_case("synth_plain_1200_450"))
    ctx = _lib.Context(0)
    ctx.load_batch(np.array([0, len(br) + len(tr)]), np.array([len(br)]), np.concatenate([bx, tx]),
                   np.concatenate([br, tr]))
    ctx.run_graph()
    v, ms = ctx.surface_variants()
    assert all(x in (0, 1, 2) for x in v)
    assert np.isfinite(ms).all() and (ms >= 0).all()
    for k in range(5):
        assert ms[k, v[k]] == ms[k].min()


def test_concurrent_dot_passes_give_identical_surfaces():
    """
    The convex / toroidal / concave passes on side streams, and the SC
    searches beside the CMS search and its adjoint (graph branches of the
    captured pipeline), give the same dots, CMS, SC and gradient as the
    passes one after the other.
    """
    from cms_cuda import _lib
    from parity import inputs, load_case
    names = ("golden_pkl", "synth_small_s7", "synth_zero_radii", "smallmol_7jkv_pdb", "sc_example_pdb")
    xyz, rad, off, nb = [], [], [0], []
    for n in names:
        bx, br, tx, tr = inputs(load_case(n))
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    X, R = np.concatenate(xyz), np.concatenate(rad)
    out = []
    modes = (0, _lib.CONC_COUNT, _lib.CONC_EMIT, _lib.CONC_READOUT, True)
    for conc in modes:
        ctx = _lib.Context(0)
        if conc is True:
            with pytest.raises(_lib.CmsError):
                ctx.set_concurrency(8)
        ctx.set_concurrency(conc)
        ctx.set_backward(True, target_side=True)
        ctx.load_batch(np.array(off), np.array(nb), X, R)
        ctx.run_graph()
        ctx.graph_launch()                 # a replay: every pass keeps and reuses its stash
        grad = ctx.grad_xyz()
        dots = []
        for c in range(len(names)):
            i = ctx.info(c)
            dots += [ctx.export_dots(c, m, i) for m in (0, 1)]
            dots.append(ctx.export_atoms(c, int(off[c + 1] - off[c])))
        pa, tot = ctx.contact_ms(per_atom=True)
        sc, sides = ctx.shape_complementarity()
        trimmed = [ctx.export_trimmed(c, m, ctx.info(c)) for c in range(len(names)) for m in (0, 1)]
        out.append((dots, pa, tot, sc, sides, grad, trimmed))
    for other in out[1:]:
        for a, b in zip(out[0][0], other[0]):
            for x, y in zip(a, b):
                assert np.array_equal(x, y, equal_nan=True)
        for k in (1, 2, 3, 4, 5):
            assert np.array_equal(out[0][k], other[k])
        for x, y in zip(out[0][6], other[6]):
            assert np.array_equal(x, y)
