"""
Batched evaluation of many independent complexes in one pass of the CUDA
pipeline (one set of launches for the whole batch, captured once in a CUDA
graph and replayed).

The reference evaluates one complex per calculator (cms-cuda/_api.py:41-133,
and the CLI's serial loop examples/calculate_cms_sc.py:130-212); this module
is the batched form of the same readouts: per complex the target- and
binder-side CMS (with per-atom arrays) and the SC triple.
"""

import numpy as np

from . import _lib


class BatchResult:
    """Per-complex outputs of one batched run."""

    def __init__(self, totals, sc, sides, per_atom=None, grad=None):
        self.cms = totals[:, 1].copy()              # target side (calculate_contact_ms)
        self.grad = grad                            # d(target-side CMS)/d(xyz) (N x 3) when requested
        self.cms_binder = totals[:, 0].copy()
        self.sc = sc[:, 0].copy()
        self.sc_area = sc[:, 1].copy()
        self.sc_distance = sc[:, 2].copy()
        self.sides = sides
        self.per_atom = per_atom


class BatchCalculator:
    """
    Holds one device context and the workspace of a batch shape.  load() the
    concatenated batch (binder atoms then target atoms per complex), then
    run().  Re-loading a batch of the same shape replays the captured graph.
    """

    def __init__(self, device=0, settings=None):
        self.ctx = _lib.Context(device)
        if settings is not None:
            self.ctx.set_settings(settings)
        self._settings = settings
        self._grad = False

    def set_settings(self, settings):
        self.ctx.set_settings(settings)
        self._settings = settings

    def load(self, atom_off, n_binder, xyz, radius, density=None):
        self.ctx.load_batch(atom_off, n_binder, xyz, radius, density)

    def run(self, graph=True, per_atom=False, grad=False, grad_out=None):
        """
        Surfaces + CMS (both sides) + SC of every loaded complex; with
        grad=True also d(target-side CMS)/d(xyz) of every atom (in the
        captured graph when graph=True), written to `grad_out` when given
        (N x 3 float64; a pinned buffer makes the read-back a direct copy).
        """
        if graph:
            if grad != self._grad:
                self.ctx.set_backward(grad, target_side=True)
                self._grad = grad
            self.ctx.run_graph()
        else:
            self.ctx.generate(all_atoms=False)
        pa, totals = self.ctx.contact_ms(per_atom=per_atom)
        sc, sides = self.ctx.shape_complementarity()
        g = None
        if grad:
            if graph:
                g = self.ctx.grad_xyz(grad_out)
            else:
                g = self.ctx.contact_ms_backward(target_side=True)
                if grad_out is not None:
                    grad_out[...] = g
                    g = grad_out
        return BatchResult(totals, sc, sides, pa if per_atom else None, g)

    def run_stream(self, batches, grad_outs):
        """
        Evaluate a sequence of batches of one shape (the same atom_off and
        n_binder) with the host<->device copies of neighbouring batches
        overlapped with the pipeline: while batch k runs, batch k+1's
        coordinates and radii upload on a copy stream, and batch k's gradient
        downloads while batch k+1 runs.  `batches` is a list of
        (atom_off, n_binder, xyz, radius) host arrays (pinned xyz / radius
        make the uploads asynchronous); `grad_outs` one pinned float64 N x 3
        host array per batch, which receives that batch's d(target-side
        CMS)/d(xyz).  Returns the BatchResult of every batch; the gradients
        are in place when it returns.
        """
        import torch
        n = check_stream_args(batches, grad_outs)
        if not self._grad:
            self.ctx.set_backward(True, target_side=True)
            self._grad = True
        dev = torch.device("cuda", self.ctx.device)
        stage_x = [torch.empty((n, 3), dtype=torch.float64, device=dev) for _ in range(2)]
        stage_r = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(2)]
        stage_g = [torch.empty((n, 3), dtype=torch.float64, device=dev) for _ in range(2)]
        copy = torch.cuda.Stream(device=dev)
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_out = [None, None]

        def upload(k):
            _, _, x, r = batches[k]
            with torch.cuda.stream(copy):
                stage_x[k % 2].copy_(torch.from_numpy(np.asarray(x, np.float64).reshape(-1, 3)), non_blocking=True)
                stage_r[k % 2].copy_(torch.from_numpy(np.asarray(r, np.float64)), non_blocking=True)
                ev_in[k % 2].record(copy)

        results = []
        upload(0)
        for k in range(len(batches)):
            off, nb = batches[k][0], batches[k][1]
            ev_in[k % 2].synchronize()
            if k + 1 < len(batches):
                upload(k + 1)            # its staging buffers were last read by batch k - 1's load
            self.ctx.load_batch_device(off, nb, stage_x[k % 2].data_ptr(), stage_r[k % 2].data_ptr())
            self.ctx.run_graph()
            _, totals = self.ctx.contact_ms(per_atom=False)
            sc, sides = self.ctx.shape_complementarity()
            if ev_out[k % 2] is not None:
                ev_out[k % 2].synchronize()      # batch k - 2's download has left this buffer
            self.ctx.grad_xyz_device(stage_g[k % 2].data_ptr())
            with torch.cuda.stream(copy):
                torch.from_numpy(grad_outs[k]).copy_(stage_g[k % 2], non_blocking=True)
                ev_out[k % 2] = torch.cuda.Event()
                ev_out[k % 2].record(copy)
            results.append(BatchResult(totals, sc, sides, None, grad_outs[k]))
        copy.synchronize()
        return results

    def statuses(self):
        return np.array([self.ctx.info(c).status for c in range(self.ctx.B)], dtype=np.int32)

    def kernel_launches(self):
        return self.ctx.kernel_launches()

    def profile_stages(self):
        return self.ctx.profile_stages()


def check_stream_args(batches, grad_outs):
    """Atom count N of a run_stream call; ValueError unless every batch has N atoms (N x 3 coordinates, N radii,
    consistent offsets) and there is one C-contiguous float64 N x 3 gradient buffer per batch."""
    if not batches:
        raise ValueError("no batches")
    if len(grad_outs) != len(batches):
        raise ValueError("one gradient buffer per batch")
    n = int(np.asarray(batches[0][0])[-1])
    for off, nb, x, r in batches:
        if int(np.asarray(off)[-1]) != n or np.shape(x) != (n, 3) or np.shape(r) != (n,) or len(nb) != len(off) - 1:
            raise ValueError("run_stream needs batches of one atom count, with N x 3 coordinates and N radii")
    for g in grad_outs:
        if g.dtype != np.float64 or g.shape != (n, 3) or not g.flags.c_contiguous:
            raise ValueError(f"each gradient buffer must be a C-contiguous float64 array of shape ({n}, 3)")
    return n


def pack(complexes):
    """Concatenate [(binder_xyz, binder_radii, target_xyz, target_radii), ...] into batch arrays."""
    xyz, rad, off, nb = [], [], [0], []
    for bx, br, tx, tr in complexes:
        bx = np.asarray(bx, np.float64).reshape(-1, 3)
        tx = np.asarray(tx, np.float64).reshape(-1, 3)
        xyz += [bx, tx]
        rad += [np.asarray(br, np.float64), np.asarray(tr, np.float64)]
        nb.append(len(bx))
        off.append(off[-1] + len(bx) + len(tx))
    return (np.array(off, np.int64), np.array(nb, np.int64), np.concatenate(xyz), np.concatenate(rad))


def calculate_batch(complexes, device=0, graph=False, per_atom=False):
    """CMS (target and binder side) and SC of every complex in one batched GPU pass."""
    calc = BatchCalculator(device)
    calc.load(*pack(complexes))
    return calc.run(graph=graph, per_atom=per_atom)
