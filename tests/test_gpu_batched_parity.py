"""
Parity of the batched workload against the reference itself: eight
complexes drawn from the 4096-complex batch (seed 2) -- the smallest, the
largest, the 10th / 50th / 90th size percentiles, the one with the largest
binder and two whose binder is a ligand-like HETATM C*/N*/O* cluster --
evaluated by the reference's CPU calculator (tests/golden/make_golden.py,
batched_4096_sample.npz) and here loaded AS ONE BATCH, through the captured
graph the benchmark replays and through the stage-synchronised path.

Dot counts, every dot's owner atom, burial flag and type, attention and
accessibility flags, neighbour counts, toroid and probe counts are exact;
CMS of both sides, per-atom CMS and the SC statistics agree within 1e-12
(reference cms-cuda/_core.py:946-1147).
"""

import numpy as np
import pytest

from parity import close, exact, load_case

pytestmark = pytest.mark.gpu

K = 8


@pytest.fixture(scope="module")
def sample():
    z = load_case("batched_4096_sample")
    cases = [{k[len(f"k{i}_"):]: v for k, v in z.items() if k.startswith(f"k{i}_")} for i in range(K)]
    return z, cases


def _batch(cases):
    off = np.zeros(len(cases) + 1, np.int64)
    off[1:] = np.cumsum([len(c["br"]) + len(c["tr"]) for c in cases])
    nb = np.array([len(c["br"]) for c in cases], np.int64)
    xyz = np.concatenate([a for c in cases for a in (c["bx"], c["tx"])])
    rad = np.concatenate([a for c in cases for a in (c["br"], c["tr"])])
    return off, nb, xyz, rad


def test_sample_covers_ligand_binders(sample):
    z, cases = sample
    assert int(np.sum(z["ligand"])) >= 2
    for c, lig in zip(cases, z["ligand"]):
        if lig:
            assert 20 <= len(c["br"]) <= 60
            assert set(np.round(c["br"], 2)) <= {1.85, 1.65, 1.60}


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "staged"])
def test_batch_matches_reference(sample, graph):
    from cms_cuda.batch import BatchCalculator
    _, cases = sample
    off, nb, xyz, rad = _batch(cases)
    bc = BatchCalculator(0)
    bc.load(off, nb, xyz, rad)
    res = bc.run(graph=graph, per_atom=True)
    ctx = bc.ctx
    for k, c in enumerate(cases):
        a0, s1, a1 = int(off[k]), int(off[k] + nb[k]), int(off[k + 1])
        i = ctx.info(k)
        assert i.status == 0
        exact(f"#{k} dot type counts", [i.convex, i.toroidal, i.concave], c["counts"])
        exact(f"#{k} probes", i.n_probes, int(c["n_probes"]))
        exact(f"#{k} toroid pairs", i.n_toroid, int(c["n_toroid"]))
        atten, access, nn, nbur = ctx.export_atoms(k, a1 - a0)
        exact(f"#{k} atten", atten, c["atten"])
        exact(f"#{k} access", access, c["access"])
        exact(f"#{k} n neighbours", nn, c["nn"])
        exact(f"#{k} n buried partners", nbur, c["nbur"])
        for m in (0, 1):
            _, _, _, bur, typ, atom = ctx.export_dots(k, m, i)
            exact(f"#{k} dots[{m}] count", len(atom), int(c[f"n_dots{m}"]))
            exact(f"#{k} dots[{m}] owner", atom, c[f"dots{m}_atom"])
            exact(f"#{k} dots[{m}] buried", bur, c[f"dots{m}_buried"])
            exact(f"#{k} dots[{m}] type", typ, c[f"dots{m}_type"])
            exact(f"#{k} trimmed[{m}] count", i.n_trimmed[m], int(c[f"n_trimmed{m}"]))
        close(f"#{k} cms target", res.cms[k], c["cms"])
        close(f"#{k} cms binder", res.cms_binder[k], c["cms_binder"])
        close(f"#{k} per-atom target", res.per_atom[s1:a1], c["per_atom_target"])
        close(f"#{k} per-atom binder", res.per_atom[a0:s1], c["per_atom_binder"])
        close(f"#{k} sc", [res.sc[k], res.sc_area[k], res.sc_distance[k]],
              [c["sc"], c["sc_area"], c["sc_distance"]])
        for m in (0, 1):
            side = res.sides[k, m]
            close(f"#{k} surface[{m}]", side[:7], c["surface"][m][:7])


def test_stream_of_batches_matches_single_runs(sample):
    """
    BatchCalculator.run_stream over three batches of one shape (the sample,
    then two rigid shifts of its binders) overlaps each batch's uploads and
    gradient download with its neighbours' pipeline runs; every batch's CMS,
    SC and gradient equal those of a plain run of that batch, bit for bit.
    """
    import torch
    from cms_cuda.batch import BatchCalculator
    _, cases = sample
    off, nb, xyz, rad = _batch(cases)
    batches = []
    for shift in (0.0, 0.37, -0.21):
        x = xyz.copy()
        for c in range(len(nb)):
            x[off[c]:off[c] + nb[c]] += shift
        xp = torch.from_numpy(x).pin_memory().numpy()
        rp = torch.from_numpy(rad.copy()).pin_memory().numpy()
        batches.append((off, nb, xp, rp))
    outs = [torch.empty((len(rad), 3), dtype=torch.float64).pin_memory().numpy() for _ in batches]
    bc = BatchCalculator(0)
    bc.load(*batches[0])
    bc.run(graph=True, grad=True)
    got = bc.run_stream(batches, outs)
    for (o, n, x, r), res, g in zip(batches, got, outs):
        ref = BatchCalculator(0)
        ref.load(o, n, x, r)
        want = ref.run(graph=True, grad=True)
        exact("stream cms", res.cms, want.cms)
        exact("stream binder cms", res.cms_binder, want.cms_binder)
        exact("stream sc", res.sc, want.sc)
        exact("stream gradient", g, want.grad)


def test_stream_rejects_other_atom_counts(sample):
    """run_stream takes batches of one atom count only (its device staging is sized once)."""
    from cms_cuda.batch import BatchCalculator
    _, cases = sample
    off, nb, xyz, rad = _batch(cases)
    off2, nb2, xyz2, rad2 = _batch(cases[:-1])
    bc = BatchCalculator(0)
    g = [np.empty((len(rad), 3)), np.empty((len(rad), 3))]
    with pytest.raises(ValueError):
        bc.run_stream([(off, nb, xyz, rad), (off2, nb2, xyz2, rad2)], g)
    with pytest.raises(ValueError):
        bc.run_stream([(off, nb, xyz, rad)], [np.empty((len(rad), 2))])
