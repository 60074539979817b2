"""
GPU tests of the FP64 adjoint of the contact molecular surface
(cms_contact_ms_backward and the cms_cuda.autograd Function).

* The adjoint's geometry code, run on plain doubles, recomputes every dot of
  every fixture bit for bit: the differentiated formula is the one that
  generated the surface.
* Central finite differences (1e-5 A steps) on perturbations that keep the
  dot topology (dot counts, burial, nearest-dot indices) agree with the
  gradient.
* Batched gradients equal the per-complex ones, the captured-graph gradient
  equals the eager one, and the torch Function returns the same gradient.
"""

import numpy as np
import pytest
from scipy.spatial.distance import cdist

from parity import ALL_CASES, exact, inputs, load_case

pytestmark = pytest.mark.gpu

H = 1e-5


def _ctx():
    from cms_cuda import _lib
    return _lib.Context(0)


def _load(ctx, cases):
    xyz, rad, off, nb = [], [], [0], []
    for c in cases:
        bx, br, tx, tr = inputs(c)
        xyz += [bx, tx]
        rad += [br, tr]
        nb.append(len(br))
        off.append(off[-1] + len(br) + len(tr))
    X = np.concatenate(xyz).astype(np.float64)
    R = np.concatenate(rad).astype(np.float64)
    ctx.load_batch(np.array(off, np.int64), np.array(nb, np.int64), X, R)
    return X, R, np.array(off, np.int64), np.array(nb, np.int64)


def _topology(ctx, B):
    """Everything the gradient holds fixed, for comparison between runs."""
    out = []
    for c in range(B):
        info = ctx.info(c)
        out.append(("counts", tuple(info.n_dots), info.convex, info.toroidal, info.concave, info.n_probes))
        side = []
        for m in (0, 1):
            coor, _, area, bur, typ, atom = ctx.export_dots(c, m, info)
            side.append((coor, bur.astype(bool)))
            out.append(("dots", m, bur.tobytes(), typ.tobytes(), atom.tobytes()))
        for m in (0, 1):
            q, r = side[m][0][side[m][1]], side[1 - m][0][side[1 - m][1]]
            if len(q) and len(r):
                out.append(("nn", m, np.argmin(cdist(r, q, "sqeuclidean"), axis=0).tobytes()))
    return out


def _cms(ctx, X, R, off, nb, side=1):
    ctx.load_batch(off, nb, X, R)
    ctx.generate(all_atoms=False)
    _, totals = ctx.contact_ms(per_atom=False)
    return totals[:, side]


@pytest.mark.parametrize("name", ALL_CASES)
def test_recompute_is_bit_exact(name):
    ctx = _ctx()
    _load(ctx, [load_case(name)])
    ctx.generate(all_atoms=False)
    info = ctx.info(0)
    for m in (0, 1):
        coor, _, area, _, _, _ = ctx.export_dots(0, m, info)
        rc, ra = ctx.recompute_dots(0, m, info)
        exact(f"{name} mol {m} recomputed coordinates", rc, coor)
        exact(f"{name} mol {m} recomputed areas", ra, area)


def _fd_check(ctx, X, R, off, nb, grad, v, side=1):
    base = _topology(ctx, len(nb))
    cp = _cms(ctx, X + H * v, R, off, nb, side)
    tp = _topology(ctx, len(nb))
    cm = _cms(ctx, X - H * v, R, off, nb, side)
    tm = _topology(ctx, len(nb))
    if not (_same(base, tp) and _same(base, tm)):
        return None
    fd = (cp.sum() - cm.sum()) / (2 * H)
    an = float((grad * v).sum())
    return fd, an


def _same(a, b):
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if len(x) != len(y) or any((p != q) if not isinstance(p, np.ndarray) else not np.array_equal(p, q)
                                   for p, q in zip(x, y)):
            return False
    return True


@pytest.mark.parametrize("name,side", [("golden_pkl", 1), ("synth_small_s7", 1), ("synth_small_s7", 0)])
def test_gradient_matches_finite_differences(name, side):
    ctx = _ctx()
    X, R, off, nb = _load(ctx, [load_case(name)])
    ctx.generate(all_atoms=False)
    ctx.contact_ms(per_atom=False)
    grad = ctx.contact_ms_backward(target_side=bool(side))
    assert np.isfinite(grad).all()
    assert np.abs(grad).max() > 0
    rng = np.random.default_rng(11)
    # single coordinates with the largest gradients, then whole-structure directions
    order = np.argsort(-np.abs(grad).reshape(-1))
    dirs = []
    for flat in order[:6]:
        v = np.zeros_like(X).reshape(-1)
        v[flat] = 1.0
        dirs.append(v.reshape(X.shape))
    for _ in range(4):
        v = rng.normal(size=X.shape)
        dirs.append(v / np.linalg.norm(v))
    checked = 0
    worst = 0.0
    for v in dirs:
        r = _fd_check(ctx, X, R, off, nb, grad, v, side)
        if r is None:
            continue                       # the step changed the topology: not comparable
        fd, an = r
        err = abs(fd - an) / max(1.0, abs(an))
        worst = max(worst, err)
        assert err < 1e-6, f"{name}: finite difference {fd!r} vs gradient {an!r} (rel {err:.3g})"
        checked += 1
    assert checked >= 6, f"only {checked} topology-preserving directions"


def test_batched_gradient_equals_single():
    names = ("golden_pkl", "synth_small_s7", "sc_example_pdb")
    cases = [load_case(n) for n in names]
    ctx = _ctx()
    X, R, off, nb = _load(ctx, cases)
    ctx.generate(all_atoms=False)
    g = np.array([0.5, -2.0, 1.25])
    gb = ctx.contact_ms_backward(True, g)
    for i, c in enumerate(cases):
        s = _ctx()
        _load(s, [c])
        s.generate(all_atoms=False)
        gs = s.contact_ms_backward(True, g[i:i + 1])
        exact(f"{names[i]} batched gradient", gb[off[i]:off[i + 1]], gs)


def test_graph_gradient_equals_eager():
    cases = [load_case(n) for n in ("golden_pkl", "synth_small_s7")]
    ctx = _ctx()
    _load(ctx, cases)
    ctx.set_backward(True, target_side=True)
    ctx.run_graph()
    g_graph = ctx.grad_xyz()
    ctx.graph_launch()
    exact("graph replay gradient", ctx.grad_xyz(), g_graph)
    e = _ctx()
    _load(e, cases)
    e.generate(all_atoms=False)
    exact("graph vs eager gradient", g_graph, e.contact_ms_backward(True))


def test_torch_function():
    import torch
    from cms_cuda import autograd
    c = load_case("synth_small_s7")
    bx, br, tx, tr = inputs(c)
    b = torch.tensor(bx, dtype=torch.float64, device="cuda", requires_grad=True)
    t = torch.tensor(tx, dtype=torch.float64, device="cuda", requires_grad=True)
    val = autograd.contact_ms(b, br, t, tr)
    (3.0 * val).backward()
    ctx = _ctx()
    _load(ctx, [c])
    ctx.generate(all_atoms=False)
    _, totals = ctx.contact_ms(per_atom=False)
    assert float(val.detach()) == totals[0, 1]
    g = ctx.contact_ms_backward(True, np.array([3.0]))
    exact("torch binder gradient", b.grad.cpu().numpy(), g[:len(br)])
    exact("torch target gradient", t.grad.cpu().numpy(), g[len(br):])


@pytest.mark.parametrize("name,side", [("golden_pkl", 1), ("synth_small_s7", 1), ("synth_small_s7", 0),
                                       ("sc_example_pdb", 1)])
def test_gradient_matches_torch_autograd(name, side):
    """The adjoint against torch FP64 autograd of the same fixed-topology formula."""
    import torch
    import torch_cms_formula as F
    c = load_case(name)
    ctx = _ctx()
    X, R, off, nb = _load(ctx, [c])
    ctx.generate(all_atoms=False)
    _, totals = ctx.contact_ms(per_atom=False)
    grad = ctx.contact_ms_backward(target_side=bool(side))
    topo = F.topology(ctx, 0)
    Xt = torch.tensor(X, dtype=torch.float64, requires_grad=True)
    for m in (0, 1):
        p, a = F.dots(Xt, R, topo["dens"], 1.7, topo, m)
        assert np.abs(p.detach().numpy() - topo["dots"][m]["coor"]).max() < 1e-9
        assert np.abs(a.detach().numpy() - topo["dots"][m]["area"]).max() < 1e-9
    cms = F.contact_ms(Xt, R, 1.7, 0.5, topo, side)
    assert abs(float(cms.detach()) - totals[0, side]) <= 1e-10 * max(1.0, abs(totals[0, side]))
    cms.backward()
    ref = Xt.grad.numpy()
    scale = max(1.0, np.abs(ref).max())
    err = np.abs(ref - grad).max() / scale
    assert err < 1e-9, f"{name} side {side}: adjoint vs torch autograd, max scaled difference {err:.3g}"
