"""
Batch CLI (cms_cuda.cli) against the single-complex entry points: structures
written as PDB files, read back by the loader, evaluated in one batch; each
row must equal calculate_contact_ms / calculate_shape_complementarity /
calculate_maximum_possible_contact_ms on the same loaded atoms (rounded as the
CLI prints them), the per-residue tables (summed on the device) must equal
the reference CLI's per-residue fold of the per-atom CMS, and a file whose
selection is empty must get an error row without stopping the others.
"""

import csv
import io
import os

import numpy as np
import pytest


def _write_structures(tmp_path, n=2):
    from cms_cuda import synth
    batch = synth.make_batch([900, 1300, 700][:n], [260, 180, 90][:n], 11, names=True)
    paths = []
    for c in range(n):
        p = str(tmp_path / f"cplx{c}.pdb")
        synth.write_pdb(p, batch, c)
        paths.append(p)
    return paths


def test_cli_requires_both_sides(tmp_path):
    from cms_cuda import cli
    with pytest.raises(SystemExit):
        cli.main([str(tmp_path / "x.pdb"), "--binder-chains", "B"], out=io.StringIO())


def test_write_pdb_round_trip(tmp_path):
    from cms_cuda import synth
    from cms_cuda.loader import load_atoms
    batch = synth.make_batch([400], [150], 5, names=True)
    p = str(tmp_path / "c.pdb")
    synth.write_pdb(p, batch, 0)
    bx, br, _ = load_atoms(p, chains="B")
    tx, tr, _ = load_atoms(p, chains="A")
    gbx, gbr, gtx, gtr = batch.complex(0)
    as_written = np.vectorize(lambda v: float(np.float32(f"{v:.3f}")))
    assert np.array_equal(bx, as_written(gbx)) and np.array_equal(tx, as_written(gtx))
    assert np.array_equal(br, gbr) and np.array_equal(tr, gtr)


@pytest.mark.gpu
def test_cli_rows_match_single_complex_api(tmp_path):
    from cms_cuda import cli
    from cms_cuda._api import (calculate_contact_ms, calculate_maximum_possible_contact_ms,
                               calculate_shape_complementarity)
    from cms_cuda.loader import load_atoms
    paths = _write_structures(tmp_path, 3)
    bad = str(tmp_path / "nobinder.pdb")
    with open(paths[0]) as src, open(bad, "w") as dst:
        dst.writelines(line for line in src if line[21:22] != "B")
    paths.insert(1, bad)
    out_csv = str(tmp_path / "rows.csv")
    per_dir = str(tmp_path / "per_residue")
    rows = cli.main(paths + ["--binder-chains", "B", "--target-chains", "A", "--max-cms",
                             "--csv", out_csv, "--per-residue", per_dir], out=io.StringIO())
    assert len(rows) == 4 and "error" in rows[1] and "error" not in rows[0]
    with open(out_csv) as f:
        assert [r["structure"] for r in csv.DictReader(f)] == [os.path.basename(p) for p in paths]
    for p, row in zip(paths, rows):
        if p == bad:
            continue
        bx, br, _ = load_atoms(p, chains="B")
        tx, tr, _ = load_atoms(p, chains="A")
        cms, per_t, calc = calculate_contact_ms(bx, br, tx, tr)
        cms_b = calc.calc_contact_molecular_surface(target_side=False)
        cms_b = cms_b[0] if isinstance(cms_b, tuple) else cms_b
        sc, area, med, _ = calculate_shape_complementarity(bx, br, tx, tr)
        mt = calculate_maximum_possible_contact_ms(tx, tr)[0]
        mb = calculate_maximum_possible_contact_ms(bx, br)[0]
        assert row["binder_atoms"] == len(bx) and row["target_atoms"] == len(tx)
        assert row["cms"] == round(float(cms), 4) and row["cms_binder"] == round(float(cms_b), 4)
        assert row["sc"] == round(float(sc), 4) and row["sc_area"] == round(float(area), 4)
        assert row["sc_median_dist"] == round(float(med), 4)
        assert row["max_cms_target"] == round(float(mt), 4) and row["max_cms_binder"] == round(float(mb), 4)
        base = os.path.splitext(os.path.basename(p))[0]
        per_b = calc.calc_contact_molecular_surface(target_side=False)[1]
        for side, chain, values in (("target", "A", per_t), ("binder", "B", per_b)):
            _, _, info = load_atoms(p, chains=chain)
            with open(os.path.join(per_dir, f"{base}_{side}_cms.csv")) as f:
                tab = list(csv.DictReader(f))
            want = _residue_fold(info, values)
            assert [(r["chain"], r["resnum"], r["resname"]) for r in tab] == list(want)
            assert [float(r["cms"]) for r in tab] == [round(v, 4) for v in want.values()]
        assert row["cms"] == pytest.approx(float(np.sum(per_t)), abs=1e-3)


def _residue_fold(info, values):
    """The reference CLI's per-residue table (examples/calculate_cms_sc.py:105-114): per (chain, resnum,
    resname) in order of first appearance, a running sum of the per-atom values from 0.0."""
    out = {}
    for rec, v in zip(info, values):
        out[rec[:3]] = out.get(rec[:3], 0.0) + float(v)
    return out


@pytest.mark.gpu
def test_device_residue_sums_exact(tmp_path):
    """Device per-residue sums equal the sequential host fold bit for bit, for every structure of a batch."""
    from cms_cuda import _lib
    from cms_cuda.loader import load_atoms, residue_groups
    paths = _write_structures(tmp_path, 3)
    sides = [(load_atoms(p, chains="B"), load_atoms(p, chains="A")) for p in paths]
    off = np.zeros(len(paths) + 1, np.int64)
    off[1:] = np.cumsum([len(b[1]) + len(t[1]) for b, t in sides])
    xyz = np.concatenate([a for b, t in sides for a in (b[0], t[0])])
    rad = np.concatenate([a for b, t in sides for a in (b[1], t[1])])
    ctx = _lib.Context(0)
    ctx.load_batch(off, np.array([len(b[1]) for b, _ in sides]), xyz, rad)
    ctx.generate(all_atoms=False)
    per_atom, _ = ctx.contact_ms(per_atom=True)
    for c, (b, t) in enumerate(sides):
        for info, first in ((b[2], off[c]), (t[2], off[c] + len(b[1]))):
            keys, roff, atoms = residue_groups(info, first)
            got = ctx.residue_sums(roff, atoms)
            want = _residue_fold(info, per_atom[first:first + len(info)])
            assert list(want) == keys
            assert np.array_equal(got, np.array(list(want.values())))
    # a map that points past the batch is rejected
    with pytest.raises(_lib.CmsError):
        ctx.residue_sums(np.array([0, 1]), np.array([len(rad)], np.int32))
