"""
GPU tests of the rigid-body pose refinement driver (cms_refine_*): the
recorded CMS of the starting poses equals a fresh evaluation, the ascent
raises the CMS, the returned coordinates are the rigid motions it reports,
and the final poses evaluate identically through the plain per-complex path.
"""

import numpy as np
import pytest

from parity import exact, inputs, load_case

pytestmark = pytest.mark.gpu


def _batch(names):
    xyz, rad, off, nb = [], [], [0], []
    for n in names:
        bx, br, tx, tr = inputs(load_case(n))
        xyz += [bx, tx]; rad += [br, tr]; nb.append(len(br)); off.append(off[-1] + len(br) + len(tr))
    return np.array(off), np.array(nb), np.concatenate(xyz), np.concatenate(rad)


def test_refinement_ascends_and_reports_consistent_poses():
    from cms_cuda import _lib, MolecularSurfaceCalculator
    from cms_cuda.refine import perturb_binders, refine_poses
    off, nb, X, R = _batch(("golden_pkl", "synth_small_s7", "sc_example_pdb"))
    X0 = perturb_binders(X, off, nb, max_deg=10.0, max_shift=1.0, seed=5)
    res = refine_poses(off, nb, X0, R, steps=40)
    # the first recorded CMS is the starting poses' CMS
    ctx = _lib.Context(0)
    ctx.load_batch(off, nb, X0, R)
    ctx.generate(all_atoms=False)
    _, tot = ctx.contact_ms(per_atom=False)
    exact("CMS of the starting poses", res.history[0], tot[:, 1])
    assert np.isfinite(res.history).all()
    assert res.history[-1].sum() > res.history[0].sum()
    # coordinates = the reported rigid motions of the starting binders; targets unchanged
    for c in range(len(nb)):
        a0, a1, n = off[c], off[c + 1], nb[c]
        b0 = X0[a0:a0 + n]
        cen = np.zeros(3)
        for k in range(3):                    # the device's centroid: a fixed-order sum, compared loosely
            cen[k] = b0[:, k].sum() / n
        want = (b0 - cen) @ res.rot[c].T + cen + res.trans[c]
        assert np.abs(res.xyz[a0:a0 + n] - want).max() < 1e-9
        exact("target atoms", res.xyz[a0 + n:a1], X0[a0 + n:a1])
        assert np.abs(res.rot[c] @ res.rot[c].T - np.eye(3)).max() < 1e-12
    # the final poses: batched evaluation == plain per-complex evaluation
    ctx.load_batch(off, nb, res.xyz, R)
    ctx.generate(all_atoms=False)
    _, tot = ctx.contact_ms(per_atom=False)
    for c in range(len(nb)):
        a0, a1, n = off[c], off[c + 1], nb[c]
        m = MolecularSurfaceCalculator(0)
        m.add_binder_and_target(res.xyz[a0:a0 + n], R[a0:a0 + n], res.xyz[a0 + n:a1], R[a0 + n:a1])
        cms, _ = m.CalcLoaded()
        assert cms == tot[c, 1]


def test_refinement_history_is_the_evaluated_poses():
    """Step k's record equals a fresh evaluation of the pose reached after k steps."""
    from cms_cuda import _lib
    from cms_cuda.refine import perturb_binders
    off, nb, X, R = _batch(("synth_small_s7", "golden_pkl"))
    X0 = perturb_binders(X, off, nb, max_deg=8.0, max_shift=1.0, seed=9)
    ctx = _lib.Context(0)
    ctx.load_batch(off, nb, X0, R)
    ctx.refine_begin(X0, 10)
    h1 = ctx.refine_run(6)
    _, _, x6 = ctx.refine_pose(xyz=True)
    h2 = ctx.refine_run(1)
    ctx.refine_end()
    e = _lib.Context(0)
    e.load_batch(off, nb, x6, R)
    e.generate(all_atoms=False)
    _, tot = e.contact_ms(per_atom=False)
    assert h1.shape == (6, 2)
    exact("CMS at step 6", h2[0], tot[:, 1])


def test_refined_poses_match_the_oracle():
    """
    Final poses of a short refinement evaluated by the CPU oracle (the
    reference's NumPy algorithm, bit-exact to it): the CMS the refinement
    recorded for its last pose, and a fresh batched evaluation, agree with the
    oracle's FP64 CMS within 1e-12, and the dot counts are identical.
    """
    from cms_cuda import _lib
    from cms_cuda.refine import perturb_binders, refine_poses
    from oracle import cms_oracle
    from parity import close
    off, nb, X, R = _batch(("golden_pkl", "synth_small_s7"))
    X0 = perturb_binders(X, off, nb, max_deg=12.0, max_shift=1.5, seed=9)
    res = refine_poses(off, nb, X0, R, steps=30)
    ctx = _lib.Context(0)
    ctx.load_batch(off, nb, res.xyz, R)
    ctx.generate(all_atoms=False)
    _, tot = ctx.contact_ms(per_atom=False)
    for c in range(len(nb)):
        a0, a1, n = off[c], off[c + 1], nb[c]
        ref = cms_oracle.run_complex(res.xyz[a0:a0 + n], R[a0:a0 + n], res.xyz[a0 + n:a1], R[a0 + n:a1], sc=False)
        close(f"complex {c} final-pose CMS vs oracle", tot[c, 1], ref["cms"])
        S = ref["surface"]
        info = ctx.info(c)
        exact(f"complex {c} dots", [info.n_dots[0], info.n_dots[1]],
              [len(S.dot_arrays[0]["area"]), len(S.dot_arrays[1]["area"])])
