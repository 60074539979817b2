"""
Differentiable contact molecular surface for PyTorch.

``batched_contact_ms`` returns the per-complex CMS of one side (the target
side by default, as ``calculate_contact_ms`` reports it) as a tensor whose
gradient with respect to the atom coordinates comes from the library's FP64
adjoint (``cms_contact_ms_backward``): dot positions and areas are
differentiated through the convex, toroidal and concave constructions and the
probe solves, with the dot topology of the forward pass held fixed -- which
dots exist, their burial, their subdivision indices, the construction branches
and each query dot's nearest dot.  The reference has no gradient; its value is
``calc_contact_molecular_surface`` (cms-cuda/_core.py:946-1004).

The context that ran the forward pass is kept until the backward pass (or
until the graph is freed), so the gradient is taken at exactly the generated
surface.
"""

import numpy as np
import torch

from . import _lib
from ._api import _device_index


class _Held:
    """A pooled context reserved from the forward pass to the backward pass."""

    def __init__(self, device):
        self.device = device
        self.ctx = _lib.acquire_context(device)

    def release(self):
        if self.ctx is not None:
            _lib.release_context(self.ctx, self.device)
            self.ctx = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class ContactMSFunction(torch.autograd.Function):
    """xyz (N, 3) float64 -> per-complex CMS (B,) of one side."""

    @staticmethod
    def forward(ctx, xyz, radius, atom_off, n_binder, target_side, device):
        held = _Held(device)
        c = held.ctx
        xyz_np = xyz.detach().to("cpu", torch.float64).contiguous().numpy()
        rad_np = np.ascontiguousarray(radius, dtype=np.float64)
        c.load_batch(atom_off, n_binder, xyz_np, rad_np)
        c.generate(all_atoms=False)
        _, totals = c.contact_ms(per_atom=False)
        side = 1 if target_side else 0
        ctx.held = held
        ctx.side = side
        return torch.from_numpy(totals[:, side].copy()).to(xyz.device)

    @staticmethod
    def backward(ctx, grad_out):
        held = ctx.held
        g = grad_out.detach().to("cpu", torch.float64).contiguous().numpy()
        grad = held.ctx.contact_ms_backward(target_side=ctx.side == 1, grad_total=g)
        held.release()
        return torch.from_numpy(grad).to(grad_out.device), None, None, None, None, None


def batched_contact_ms(xyz, radius, atom_off, n_binder, target_side=True, device="auto"):
    """
    Per-complex CMS (B,) of the concatenated batch (per complex: binder atoms,
    then target atoms; ``atom_off`` (B + 1) and ``n_binder`` (B) as for
    ``cms_cuda.batch.BatchCalculator.load``), differentiable with respect to
    ``xyz`` (N, 3), a float64 tensor on any device.
    """
    dev = _device_index(device)
    radius = radius.detach().cpu().numpy() if isinstance(radius, torch.Tensor) else np.asarray(radius)
    return ContactMSFunction.apply(xyz, radius, np.asarray(atom_off, np.int64), np.asarray(n_binder, np.int64),
                                   bool(target_side), dev)


def contact_ms(binder_xyz, binder_radii, target_xyz, target_radii, target_side=True, device="auto"):
    """
    CMS of one complex as a 0-d tensor, differentiable with respect to
    ``binder_xyz`` and ``target_xyz`` (float64 tensors), the counterpart of
    ``calculate_contact_ms`` (cms-cuda/_api.py:41-72).
    """
    xyz = torch.cat([binder_xyz.reshape(-1, 3), target_xyz.reshape(-1, 3)], 0)
    rad = np.concatenate([np.asarray(binder_radii, np.float64).reshape(-1), np.asarray(target_radii, np.float64).reshape(-1)])
    nb = int(binder_xyz.reshape(-1, 3).shape[0])
    out = batched_contact_ms(xyz, rad, [0, len(rad)], [nb], target_side, device)
    return out[0]
