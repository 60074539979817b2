"""
Batch command line: contact molecular surface (CMS) and shape
complementarity (SC) of many complex structures (PDB or mmCIF) in one GPU
batch.

The command-line contract is the reference example CLI's
(examples/calculate_cms_sc.py:130-211): the same options, the same
``key=value`` rows (structure, device, atom counts, cms, cms_binder, sc,
sc_area, sc_median_dist, max_cms_*, cms_fraction_*, seconds; or structure and
error), the same CSV columns and per-residue tables
``<structure>_<side>_cms.csv`` (chain, resnum, resname, cms).  The work is
organised differently: every loadable structure of the command line goes into
one batched pass of the CUDA pipeline (plus one all-atoms batch for
``--max-cms``), and the per-residue tables are summed on the device for the
whole batch at once.  A structure that cannot be loaded gets an error row and
the others proceed; ``seconds`` is the batch's wall time divided evenly
between its structures.

  python -m cms_cuda.cli designs/*.pdb --binder-chains B --target-chains A \\
      --csv cms_sc.csv --per-residue per_residue/ --max-cms
"""

import argparse
import csv
import os
import sys
import time

import numpy as np

from .loader import load_atoms, residue_groups

SIDES = ("binder", "target")
ROUND = 4          # decimals of every printed / written value


def _names(text):
    """'A,B,,C' -> ['A', 'B', 'C']; None / '' -> None."""
    items = [t for t in (text or "").split(",") if t]
    return items or None


class Selection:
    """Which atoms of a structure form one side (the loader's keyword arguments)."""

    def __init__(self, chains=None, resnames=None, exclude=None, keep_water=False, keep_ions=False):
        self.kwargs = dict(chains=chains, resnames=set(resnames) if resnames else None,
                           exclude_resnames=set(exclude or ()), keep_water=keep_water, keep_ions=keep_ions)
        self.defined = bool(chains or resnames)

    @classmethod
    def from_args(cls, args, side):
        return cls(_names(getattr(args, f"{side}_chains")), _names(getattr(args, f"{side}_resnames")),
                   _names(getattr(args, f"{side}_exclude")), args.keep_water, args.keep_ions)

    def load(self, path):
        return load_atoms(path, **self.kwargs)


class Loaded:
    """One structure's two sides as loaded: coordinates, radii and per-atom records."""

    def __init__(self, slot, name, sides):
        self.slot, self.name = slot, name
        (self.bx, self.br, self.binfo), (self.tx, self.tr, self.tinfo) = sides

    def invisible_atoms(self):
        """Per side: (count, sample of (residue, atom) names) of atoms with no radius-table entry."""
        out = {}
        for side, radii, info in (("binder", self.br, self.binfo), ("target", self.tr, self.tinfo)):
            zero = np.nonzero(radii == 0.0)[0]
            if len(zero):
                out[side] = (len(zero), sorted({(info[a][2], info[a][3]) for a in zero}))
        return out


def parser():
    ap = argparse.ArgumentParser(prog="python -m cms_cuda.cli", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("structures", nargs="+", help="structure files (.pdb / .ent / .cif / .mmcif), one complex each")
    for side in SIDES:
        ap.add_argument(f"--{side}-chains", metavar="IDS",
                        help=f"chains forming the {side}, comma-separated (all chains if not given)")
        ap.add_argument(f"--{side}-resnames", metavar="NAMES",
                        help=f"restrict the {side} to residues with these names, comma-separated")
        ap.add_argument(f"--{side}-exclude", metavar="NAMES",
                        help=f"leave residues with these names out of the {side}, comma-separated")
    ap.add_argument("--keep-water", action="store_true", help="do not drop water residues")
    ap.add_argument("--keep-ions", action="store_true",
                    help="do not drop one-atom hetero residues (ions; most have no radius and stay invisible)")
    ap.add_argument("--device", default="auto", help="auto, cuda, gpu or cuda:N (there is no CPU path)")
    ap.add_argument("--no-sc", action="store_true", help="report CMS only, no shape complementarity")
    ap.add_argument("--max-cms", action="store_true",
                    help="add each side's maximum possible CMS (its whole molecular surface area)")
    ap.add_argument("--csv", metavar="FILE", help="also write the rows, one per structure, as CSV")
    ap.add_argument("--per-residue", metavar="DIR", help="write a per-residue CMS table per structure and side")
    return ap


def _pack(loaded):
    """Batch arrays: per complex its binder atoms, then its target atoms."""
    n_binder = np.array([len(L.br) for L in loaded], np.int64)
    atom_off = np.zeros(len(loaded) + 1, np.int64)
    atom_off[1:] = np.cumsum([len(L.br) + len(L.tr) for L in loaded])
    xyz = np.concatenate([a for L in loaded for a in (L.bx, L.tx)])
    rad = np.concatenate([a for L in loaded for a in (L.br, L.tr)])
    return atom_off, n_binder, xyz, rad


def _residue_tables(ctx, loaded, atom_off):
    """Per structure and side: [(chain, resnum, resname, summed per-atom CMS)], summed on the device."""
    parts, offs, atoms, base = [], [np.zeros(1, np.int64)], [], 0
    for c, L in enumerate(loaded):
        for side, info, first in (("target", L.tinfo, atom_off[c] + len(L.br)), ("binder", L.binfo, atom_off[c])):
            keys, off, members = residue_groups(info, first)
            parts.append((c, side, keys))
            offs.append(off[1:] + base)
            atoms.append(members)
            base += len(members)
    sums = ctx.residue_sums(np.concatenate(offs), np.concatenate(atoms))
    tables, r = {}, 0
    for c, side, keys in parts:
        tables[(c, side)] = [(*k, float(v)) for k, v in zip(keys, sums[r:r + len(keys)])]
        r += len(keys)
    return tables


def _max_cms(dev, loaded):
    """Maximum possible CMS of every target and binder (each alone as molecule 0, all atoms attended)."""
    from . import _lib
    alone = [(L.tx, L.tr) for L in loaded] + [(L.bx, L.br) for L in loaded]
    off = np.zeros(len(alone) + 1, np.int64)
    off[1:] = np.cumsum([len(r) for _, r in alone])
    ctx = _lib.Context(dev)
    ctx.load_batch(off, np.diff(off), np.concatenate([x for x, _ in alone]), np.concatenate([r for _, r in alone]))
    ctx.generate(all_atoms=True)
    totals = ctx.max_contact_ms()[1]
    return totals[:len(loaded)], totals[len(loaded):]


def evaluate(loaded, dev, sc=True, max_cms=False, per_residue=False):
    """
    One batched pass over the loaded structures: a result dict per structure
    (its row values, or an error), plus per-residue tables when asked.
    """
    from . import _lib
    atom_off, n_binder, xyz, rad = _pack(loaded)
    ctx = _lib.Context(dev)
    ctx.load_batch(atom_off, n_binder, xyz, rad)
    ctx.generate(all_atoms=False)
    infos = [ctx.info(c) for c in range(len(loaded))]
    _, totals = ctx.contact_ms(per_atom=False)
    sc_out = ctx.shape_complementarity()[0] if sc else None
    max_t, max_b = _max_cms(dev, loaded) if max_cms else (None, None)
    tables = _residue_tables(ctx, loaded, atom_off) if per_residue else {}
    results = []
    for c, L in enumerate(loaded):
        i = infos[c]
        if i.status & _lib.ST_COINCIDENT:
            results.append(dict(error=f"Coincident atoms: {i.coincident_i}:: == {i.coincident_j}::"))
            continue
        res = dict(cms=float(totals[c, 1]), cms_binder=float(totals[c, 0]))
        if sc_out is not None:
            res.update(sc=float(sc_out[c, 0]), sc_area=float(sc_out[c, 1]), sc_median_dist=float(sc_out[c, 2]))
        if max_t is not None:
            res.update(max_cms_target=float(max_t[c]), max_cms_binder=float(max_b[c]))
        res["residues"] = {side: tables.get((c, side)) for side in ("target", "binder")}
        results.append(res)
    return results


def _row(L, dev, res, seconds):
    """The printed / CSV row of one evaluated structure (the reference CLI's keys, values rounded)."""
    if "error" in res:
        return dict(structure=L.name, error=res["error"])
    row = dict(structure=L.name, device=f"cuda:{dev}", binder_atoms=len(L.br), target_atoms=len(L.tr),
               cms=round(res["cms"], ROUND), cms_binder=round(res["cms_binder"], ROUND))
    if "sc" in res:
        row.update({k: round(res[k], ROUND) for k in ("sc", "sc_area", "sc_median_dist")})
    if "max_cms_target" in res:
        mt, mb = res["max_cms_target"], res["max_cms_binder"]
        row.update(max_cms_target=round(mt, ROUND), max_cms_binder=round(mb, ROUND),
                   cms_fraction_target=round(res["cms"] / mt, ROUND) if mt else 0.0,
                   cms_fraction_binder=round(res["cms_binder"] / mb, ROUND) if mb else 0.0)
    row["seconds"] = round(seconds, 3)
    return row


def write_residue_table(path, table):
    with open(path, "w", newline="") as f:
        out = csv.writer(f)
        out.writerow(("chain", "resnum", "resname", "cms"))
        for chain, resnum, resname, value in table:
            out.writerow((chain, resnum, resname, round(value, ROUND)))


def write_rows_csv(path, rows):
    columns = list(dict.fromkeys(k for row in rows for k in row))
    with open(path, "w", newline="") as f:
        out = csv.DictWriter(f, fieldnames=columns)
        out.writeheader()
        out.writerows(rows)


def main(argv=None, out=sys.stdout):
    ap = parser()
    args = ap.parse_args(argv)
    selections = [Selection.from_args(args, side) for side in SIDES]
    if not all(s.defined for s in selections):
        ap.error("both sides need a selection, e.g. --binder-chains B --target-chains A")
    from ._api import _device_index
    dev = _device_index(args.device)
    if args.per_residue:
        os.makedirs(args.per_residue, exist_ok=True)

    start = time.perf_counter()
    rows = [None] * len(args.structures)
    loaded = []
    for slot, path in enumerate(args.structures):
        name = os.path.basename(path)
        try:
            sides = [sel.load(path) for sel in selections]
            if any(len(radii) == 0 for _, radii, _ in sides):
                raise ValueError("empty selection (binder %d atoms, target %d atoms)"
                                 % (len(sides[0][1]), len(sides[1][1])))
        except Exception as exc:           # one bad file does not stop the batch
            rows[slot] = dict(structure=name, error=str(exc))
            print(f"  error: {name}: {exc}", file=sys.stderr)
            continue
        L = Loaded(slot, name, sides)
        for side, (count, names) in L.invisible_atoms().items():
            print(f"  warning: {name} {side}: {count} atom(s) without a radius-table entry get radius 0 and add "
                  f"no surface: {names[:8]}", file=sys.stderr)
        loaded.append(L)

    if loaded:
        results = evaluate(loaded, dev, sc=not args.no_sc, max_cms=args.max_cms,
                           per_residue=bool(args.per_residue))
        seconds = (time.perf_counter() - start) / len(loaded)
        for L, res in zip(loaded, results):
            rows[L.slot] = _row(L, dev, res, seconds)
            if args.per_residue and "error" not in res:
                stem = os.path.splitext(L.name)[0]
                for side in ("target", "binder"):
                    write_residue_table(os.path.join(args.per_residue, f"{stem}_{side}_cms.csv"),
                                        res["residues"][side])
    for row in rows:
        print("  ".join(f"{k}={v}" for k, v in row.items()), file=out)
    if args.csv:
        write_rows_csv(args.csv, rows)
        print(f"wrote {args.csv}", file=out)
    return rows


if __name__ == "__main__":
    main()
