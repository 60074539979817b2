"""
Batch command line: contact molecular surface (CMS) and shape
complementarity (SC) of many complex structures (PDB or mmCIF) in one GPU
batch.

Same arguments, printed rows, CSV columns and per-residue tables as the
reference's example CLI (examples/calculate_cms_sc.py), but every structure
of the command line is evaluated in one batched pass of the CUDA pipeline
instead of one calculator per file; a structure that cannot be loaded gets an
error row and the others proceed.  "seconds" is the batch's wall time shared
equally between its structures.

  python -m cms_cuda.cli designs/*.pdb --binder-chains B --target-chains A \\
      --csv cms_sc.csv --per-residue per_residue/ --max-cms
"""

import argparse
import csv
import os
import sys
import time

import numpy as np

from .loader import load_atoms, per_residue


def _split(s):
    return [x for x in s.split(",") if x] if s else None


def _unmatched(info, radii):
    return sorted({(i[2], i[3]) for i, r in zip(info, radii) if r == 0.0})


def parser():
    ap = argparse.ArgumentParser(prog="python -m cms_cuda.cli", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("structures", nargs="+", help="PDB / mmCIF files of the complexes")
    for side in ("binder", "target"):
        ap.add_argument(f"--{side}-chains", help=f"comma-separated chain IDs of the {side} (default: all)")
        ap.add_argument(f"--{side}-resnames", help=f"only these residue names in the {side}, e.g. BTN")
        ap.add_argument(f"--{side}-exclude", help=f"residue names to drop from the {side}, e.g. BTN")
    ap.add_argument("--keep-water", action="store_true", help="keep water molecules")
    ap.add_argument("--keep-ions", action="store_true", help="keep single-atom ions (most get radius 0)")
    ap.add_argument("--device", default="auto", help="auto, cuda, gpu or cuda:N (no CPU path)")
    ap.add_argument("--no-sc", action="store_true", help="skip shape complementarity")
    ap.add_argument("--max-cms", action="store_true",
                    help="also compute the maximum possible CMS (total molecular surface) of each side")
    ap.add_argument("--csv", help="write one row per structure to this CSV file")
    ap.add_argument("--per-residue", metavar="DIR", help="write per-residue CMS tables to this directory")
    return ap


def main(argv=None, out=sys.stdout):
    ap = parser()
    args = ap.parse_args(argv)
    if not (args.binder_chains or args.binder_resnames) or not (args.target_chains or args.target_resnames):
        ap.error("select both sides, e.g. --binder-chains B --target-chains A")
    from . import _lib
    from ._api import _device_index
    dev = _device_index(args.device)

    def sel(side):
        return dict(chains=_split(getattr(args, f"{side}_chains")),
                    resnames=set(_split(getattr(args, f"{side}_resnames")) or []) or None,
                    exclude_resnames=set(_split(getattr(args, f"{side}_exclude")) or []),
                    keep_water=args.keep_water, keep_ions=args.keep_ions)

    if args.per_residue:
        os.makedirs(args.per_residue, exist_ok=True)
    t0 = time.perf_counter()
    loaded, rows = [], [None] * len(args.structures)
    for k, path in enumerate(args.structures):
        name = os.path.basename(path)
        try:
            bx, br, binfo = load_atoms(path, **sel("binder"))
            tx, tr, tinfo = load_atoms(path, **sel("target"))
            if len(bx) == 0 or len(tx) == 0:
                raise ValueError(f"empty selection (binder {len(bx)} atoms, target {len(tx)} atoms)")
            for side, info, radii in (("binder", binfo, br), ("target", tinfo, tr)):
                bad = _unmatched(info, radii)
                if bad:
                    print(f"  warning: {name} {side}: {int((radii == 0).sum())} atoms have radius 0 "
                          f"(no entry in the radius table, they are invisible): {bad[:8]}", file=sys.stderr)
            loaded.append((k, name, bx, br, binfo, tx, tr, tinfo))
        except Exception as exc:
            rows[k] = dict(structure=name, error=str(exc))
            print(f"  error: {name}: {exc}", file=sys.stderr)

    if loaded:
        # one batch: per complex the binder atoms, then the target atoms
        off = np.zeros(len(loaded) + 1, np.int64)
        nb = np.array([len(L[2]) for L in loaded], np.int64)
        off[1:] = np.cumsum([len(L[2]) + len(L[5]) for L in loaded])
        xyz = np.concatenate([np.concatenate([L[2], L[5]]) for L in loaded])
        rad = np.concatenate([np.concatenate([L[3], L[6]]) for L in loaded])
        ctx = _lib.Context(dev)
        ctx.load_batch(off, nb, xyz, rad)
        ctx.generate(all_atoms=False)
        statuses = [ctx.info(c).status for c in range(len(loaded))]
        per_atom, tot = ctx.contact_ms(per_atom=True)
        sc = ctx.shape_complementarity()[0] if not args.no_sc else None
        mx = None
        if args.max_cms:
            # maximum possible CMS: each side alone as molecule 0, all atoms attended
            sides = [(L[5], L[6]) for L in loaded] + [(L[2], L[3]) for L in loaded]
            moff = np.zeros(len(sides) + 1, np.int64)
            moff[1:] = np.cumsum([len(s[1]) for s in sides])
            m = _lib.Context(dev)
            m.load_batch(moff, np.diff(moff), np.concatenate([s[0] for s in sides]),
                         np.concatenate([s[1] for s in sides]))
            m.generate(all_atoms=True)
            mx = m.max_contact_ms()[1]
        share = (time.perf_counter() - t0) / len(loaded)
        for c, (k, name, bx, br, binfo, tx, tr, tinfo) in enumerate(loaded):
            if statuses[c] & _lib.ST_COINCIDENT:
                i = ctx.info(c)
                rows[k] = dict(structure=name, error=f"Coincident atoms: {i.coincident_i}:: == {i.coincident_j}::")
                continue
            a0, n = int(off[c]), len(bx)
            cms, cms_b = float(tot[c, 1]), float(tot[c, 0])
            row = dict(structure=name, device=f"cuda:{dev}", binder_atoms=len(bx), target_atoms=len(tx),
                       cms=round(cms, 4), cms_binder=round(cms_b, 4))
            if sc is not None:
                row.update(sc=round(float(sc[c, 0]), 4), sc_area=round(float(sc[c, 1]), 4),
                           sc_median_dist=round(float(sc[c, 2]), 4))
            if mx is not None:
                max_t, max_b = float(mx[c]), float(mx[len(loaded) + c])
                row.update(max_cms_target=round(max_t, 4), max_cms_binder=round(max_b, 4),
                           cms_fraction_target=round(cms / max_t, 4) if max_t else 0.0,
                           cms_fraction_binder=round(cms_b / max_b, 4) if max_b else 0.0)
            row["seconds"] = round(share, 3)
            if args.per_residue:
                base = os.path.splitext(name)[0]
                pa_t = per_atom[a0 + n:int(off[c + 1])]
                pa_b = per_atom[a0:a0 + n]
                for side, info, values in (("target", tinfo, pa_t), ("binder", binfo, pa_b)):
                    with open(os.path.join(args.per_residue, f"{base}_{side}_cms.csv"), "w", newline="") as f:
                        w = csv.writer(f)
                        w.writerow(["chain", "resnum", "resname", "cms"])
                        w.writerows((ch, nr, rn, round(v, 4)) for ch, nr, rn, v in per_residue(info, values))
            rows[k] = row
    for row in rows:
        print("  ".join(f"{k}={v}" for k, v in row.items()), file=out)
    if args.csv:
        keys = []
        for r in rows:
            keys += [k for k in r if k not in keys]
        with open(args.csv, "w", newline="") as f:
            w = csv.DictWriter(f, fieldnames=keys)
            w.writeheader()
            w.writerows(rows)
        print(f"wrote {args.csv}", file=out)
    return rows


if __name__ == "__main__":
    main()
