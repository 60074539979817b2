"""
Batched rigid-body pose refinement on the contact molecular surface.

Each binder moves as a rigid body (rotation about its starting centroid,
translation) by gradient ascent on its complex's target-side CMS, using the
library's FP64 adjoint; every step regenerates the surfaces in one captured
graph (cms_refine_* in the C ABI).  The reference computes CMS for fixed
coordinates only (cms-cuda/_core.py:946-1004); this is the design-loop caller
built on it.
"""

import time

import numpy as np

from . import _lib


class RefineResult:
    def __init__(self, history, rot, trans, xyz, seconds):
        self.history = history                 # (steps, B): CMS of every evaluated pose
        self.rot, self.trans, self.xyz = rot, trans, xyz
        self.seconds = seconds
        self.steps = history.shape[0]

    @property
    def initial(self):
        return self.history[0]

    @property
    def best(self):
        return self.history.max(axis=0)

    @property
    def steps_per_s(self):
        return self.steps / self.seconds if self.seconds > 0 else float("nan")


def random_rotation(rng, max_deg):
    """Rotation by a uniform angle in [0, max_deg] about a uniformly random axis."""
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    th = np.deg2rad(rng.uniform(0.0, max_deg))
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * (K @ K)


def perturb_binders(xyz, atom_off, n_binder, max_deg=15.0, max_shift=2.0, seed=0):
    """Starting poses: each binder rotated about its centroid by up to max_deg
    and shifted by up to max_shift A (uniform direction)."""
    rng = np.random.default_rng(seed)
    out = np.array(xyz, dtype=np.float64, copy=True)
    for c in range(len(n_binder)):
        a0, nb = int(atom_off[c]), int(n_binder[c])
        b = out[a0:a0 + nb]
        cen = b.mean(axis=0)
        R = random_rotation(rng, max_deg)
        d = rng.normal(size=3)
        d *= rng.uniform(0.0, max_shift) / np.linalg.norm(d)
        out[a0:a0 + nb] = (b - cen) @ R.T + cen + d
    return out


def refine_poses(atom_off, n_binder, xyz, radius, steps=200, eta_t=0.002, eta_w=0.0002, max_t=0.05,
                 max_w=np.deg2rad(0.5), device=0, ctx=None):
    """
    Run `steps` ascent steps on every complex of the batch (binder atoms
    first in each complex).  Returns a RefineResult; history[k] is the CMS of
    the poses evaluated at step k (history[0]: the starting poses).
    """
    own = ctx is None
    if own:
        ctx = _lib.Context(device)
    ctx.load_batch(atom_off, n_binder, xyz, radius)
    ctx.refine_begin(xyz, steps)
    ctx.refine_set_params(eta_t, eta_w, max_t, max_w)
    ctx.refine_run(0)                          # size, tune and capture outside the timed steps
    t0 = time.perf_counter()
    hist = ctx.refine_run(steps)
    dt = time.perf_counter() - t0
    rot, tr, x = ctx.refine_pose(xyz=True)
    ctx.refine_end()
    return RefineResult(hist, rot, tr, x, dt)
