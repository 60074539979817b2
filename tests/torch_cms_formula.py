"""
Plain torch FP64 restatement of the contact molecular surface with the dot
topology held fixed, for checking the CUDA adjoint with torch autograd.

Inputs are the atom coordinates (a tensor that may require grad) and the
topology of one generated complex as the library exports it: the frame atom
of each atom (its first neighbour), the toroid pairs, the probes (reference
order: "+" probes of both molecules, then "-" probes), and per dot its type,
unit and sub index (cms_export_dot_units), burial and the nearest-dot choice
of every query dot.  Dots are rebuilt from the atoms with the formulas of the
reference (cms-cuda/_core.py):

  convex     generate_convex_surface          _core.py:1646-1840
  toroidal   generate_toroidal_surface        _core.py:1847-2067
  concave    vec_third_loop probe solve       _core.py:1445-1643
             + generate_concave_surface       _core.py:2069-2333
  arcs       vec_sub_arc / vec_sub_div / vec_sub_cir  _core.py:2380-2527
  CMS        calc_contact_molecular_surface   _core.py:946-1004

Branches and subdivision counts are evaluated on detached values.  This is
test infrastructure only.
"""

import math

import numpy as np
import torch

TWO_PI = 6.283185307179586
MAX_SUBDIV = 100


def dot_seq(a, b):
    return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]


def dot_alt(a, b):
    return (a[:, 0] * b[:, 0] + a[:, 2] * b[:, 2]) + a[:, 1] * b[:, 1]


def norm(a):
    return torch.sqrt(dot_seq(a, a))


def normalize(a):
    return a / norm(a)[:, None]


def cross(a, b):
    return torch.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                        a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                        a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)


def count(delta, angle):
    """vec_sub_div: number of i < 100 with delta*(i+0.5) <= angle."""
    delta = np.asarray(delta, np.float64)
    angle = np.asarray(angle, np.float64)
    n = np.zeros(delta.shape, np.int64)
    for i in range(MAX_SUBDIV):
        n += (n == i) & (delta * (i + 0.5) <= angle)
    return n


def circle_frame(axis_in):
    axis = normalize(axis_in)
    v1 = torch.stack([axis[:, 1] * axis[:, 1] + axis[:, 2] * axis[:, 2],
                      axis[:, 0] * axis[:, 0] + axis[:, 2] * axis[:, 2],
                      axis[:, 0] * axis[:, 0] + axis[:, 1] * axis[:, 1]], 1)
    v1 = normalize(v1)
    sw = (dot_seq(v1, axis).detach().abs() > 0.99)[:, None]
    v1 = torch.where(sw, torch.tensor([1.0, 0.0, 0.0], dtype=v1.dtype), v1)
    v2 = normalize(cross(axis, v1))
    x = normalize(cross(axis, v2))
    return x, cross(axis, x)


def arc_angle(axis, x, v):
    y = cross(axis, x)
    ang = torch.atan2(dot_seq(v, y), dot_seq(v, x))
    ang = torch.where(ang.detach() < 0, ang + TWO_PI, ang)
    return ang, y


def sub_point(cen, rad, x, y, delta, i):
    a = delta * (i + 0.5)
    return (cen + x * (rad * torch.cos(a))[:, None]) + y * (rad * torch.sin(a))[:, None]


def _safe(t, ok, fill=1.0):
    return torch.where(ok, t, torch.full_like(t, fill))


def convex_dots(X, R, dens, rp, frame, g, sub):
    l = torch.as_tensor(sub >> 16, dtype=torch.float64)
    i = torch.as_tensor(sub & 0xFFFF, dtype=torch.float64)
    xi, xn = X[g], X[frame[g]]
    ri = torch.as_tensor(R[g]); rj = torch.as_tensor(R[frame[g]]); de = torch.as_tensor(dens[g])
    eri, erj = ri + rp, rj + rp
    north = normalize(xi - xn)
    vt = normalize(torch.stack([north[:, 1] * north[:, 1] + north[:, 2] * north[:, 2],
                                north[:, 0] * north[:, 0] + north[:, 2] * north[:, 2],
                                north[:, 0] * north[:, 0] + north[:, 1] * north[:, 1]], 1))
    sw = (dot_seq(vt, north).detach().abs() > 0.99)[:, None]
    vt = torch.where(sw, torch.tensor([1.0, 0.0, 0.0], dtype=vt.dtype), vt)
    eq = normalize(cross(north, vt))
    vql = cross(eq, north)
    dij = norm(xn - xi)
    uij = (xn - xi) / dij[:, None]
    asymm = (eri * eri - erj * erj) / dij
    tij = ((xi + xn) * 0.5) + uij * (asymm * 0.5)[:, None]
    far = (eri + erj) * (eri + erj) - dij * dij
    rd = ri - rj
    cont = dij * dij - rd * rd
    ok = (far.detach() > 0) & (cont.detach() > 0)
    rij = ((0.5 * torch.sqrt(_safe(far, ok))) * torch.sqrt(_safe(cont, ok))) / dij
    south = torch.where(ok[:, None], ((tij + vql * rij[:, None]) - xi) / eri[:, None],
                        torch.tensor([0.0, 0.0, -1.0], dtype=xi.dtype))
    ang, ylat = arc_angle(eq, north, south)
    dl = 1.0 / (torch.sqrt(de) * ri)
    nl = torch.as_tensor(count(dl.numpy(), ang.detach().numpy()), dtype=torch.float64)
    cs = (ri * ang) / nl
    fx, fy = circle_frame(north)
    lat = sub_point(torch.zeros_like(xi), ri, north, ylat, dl, l)
    dt = dot_seq(lat, north)
    cen = xi + north * dt[:, None]
    rad = torch.sqrt(ri * ri - dt * dt)
    delta = 1.0 / (torch.sqrt(de) * rad)
    nc = torch.as_tensor(count(delta.detach().numpy(), np.full(len(g), TWO_PI)), dtype=torch.float64)
    area = ((rad * TWO_PI) / nc) * cs
    return sub_point(cen, rad, fx, fy, delta, i), area


def toroidal_dots(X, R, dens, rp, a1, a2, q, sub):
    s = torch.as_tensor(sub >> 16, dtype=torch.float64)
    arc2 = torch.as_tensor(((sub >> 15) & 1) == 1)[:, None]
    t = torch.as_tensor(sub & 0x7FFF, dtype=torch.float64)
    i, j = a1[q], a2[q]
    xi, xj = X[i], X[j]
    ri, rj = torch.as_tensor(R[i]), torch.as_tensor(R[j])
    eri, erj = ri + rp, rj + rp
    diff = xj - xi
    dij_sq = dot_alt(diff, diff)
    dij = torch.sqrt(dij_sq)
    asymm = (eri * eri - erj * erj) / dij
    between = (asymm.detach().abs() < dij.detach())
    uij = diff / dij[:, None]
    tij = ((xi + xj) * 0.5) + uij * (asymm * 0.5)[:, None]
    far = (eri + erj) * (eri + erj) - dij_sq
    cont = dij_sq - (ri - rj) * (ri - rj)
    rij = ((0.5 * torch.sqrt(far)) * torch.sqrt(cont)) / dij
    density = (torch.as_tensor(dens[i]) + torch.as_tensor(dens[j])) * 0.5
    rci = (rij * ri) / eri
    rcj = (rij * rj) / erj
    rbt = rij - rp
    rb = torch.where(rbt.detach() < 0, torch.zeros_like(rbt), rbt)
    rs = ((rci + 2.0 * rb) + rcj) * 0.25
    e = rs / rij
    edens = (e * e) * density
    fx, fy = circle_frame(uij)
    dtor = 1.0 / (torch.sqrt(edens) * rij)
    ns = torch.as_tensor(count(dtor.detach().numpy(), np.full(len(q), TWO_PI)), dtype=torch.float64)
    ts = (rij * TWO_PI) / ns
    darc = 1.0 / (torch.sqrt(density) * rp)
    pij = sub_point(tij, rij, fx, fy, dtor, s)
    pi = (xi - pij) / eri[:, None]
    pj = (xj - pij) / erj[:, None]
    axis = normalize(cross(pi, pj))
    dtq = rp * rp - rij * rij
    cusp = ((dtq.detach() > 0) & between)[:, None]
    qij = tij - uij * torch.sqrt(_safe(dtq, cusp[:, 0]))[:, None]
    mid = normalize(pi + pj)
    pqi = torch.where(cusp, (qij - pij) / rp, mid)
    pqj = torch.where(cusp, torch.zeros_like(mid), mid)
    x = torch.where(arc2, pqj, pi)
    v = torch.where(arc2, pj, pqi)
    ang, y = arc_angle(axis, x, v)
    n = torch.as_tensor(count(darc.detach().numpy(), ang.detach().numpy()), dtype=torch.float64)
    ps = (rp * ang) / n
    pt = sub_point(pij, torch.full_like(rij, rp), x, y, darc, t)
    vec = pt - tij
    dtv = dot_seq(vec, uij)
    d2 = dot_seq(vec, vec) - dtv * dtv
    dist = torch.sqrt(torch.where(d2.detach() < 0, torch.zeros_like(d2), d2))
    return pt, ((ps * ts) * dist) / rij


def probe_solve(X, R, rp, i, j, k, sg):
    xi, xj, xk = X[i], X[j], X[k]
    eri = torch.as_tensor(R[i]) + rp
    erj = torch.as_tensor(R[j]) + rp
    erk = torch.as_tensor(R[k]) + rp
    diff = xj - xi
    dij = torch.sqrt(dot_alt(diff, diff))
    uij = diff / dij[:, None]
    tij = ((xi + xj) * 0.5) + uij * ((eri * eri - erj * erj) / dij * 0.5)[:, None]
    vk = xk - xi
    dik = norm(vk)
    uik = vk / dik[:, None]
    dt = dot_alt(uij, uik)
    wijk = torch.acos(torch.clamp(dt, -1.0, 1.0))
    swijk = torch.sin(wijk)
    uijk = cross(uij, uik) / swijk[:, None]
    utb = cross(uijk, uij)
    asymm = (eri * eri - erk * erk) / dik
    tik = (xi + xk) * 0.5 + uik * (asymm * 0.5)[:, None]
    dtb = dot_alt(uik, tik - tij)
    bijk = tij + utb * (dtb / swijk)[:, None]
    bma = bijk - xi
    h = torch.sqrt(eri * eri - dot_alt(bma, bma))
    sg = torch.as_tensor(sg)
    return bijk + uijk * (h * sg)[:, None], uijk * sg[:, None]


def concave_dots(X, R, dens, rp, pa, plus, p, sub):
    l = torch.as_tensor(sub >> 16, dtype=torch.float64)
    i = torch.as_tensor(sub & 0xFFFF, dtype=torch.float64)
    a0, a1, a2 = pa[0][p], pa[1][p], pa[2][p]
    pl = plus[p]
    ii = np.where(pl, a0, a1)
    jj = np.where(pl, a1, a0)
    pijk, alt = probe_solve(X, R, rp, ii, jj, a2, np.where(pl, 1.0, -1.0))
    density = ((torch.as_tensor(dens[a0]) + torch.as_tensor(dens[a1])) + torch.as_tensor(dens[a2])) / 3.0
    vp = [normalize(X[a] - pijk) for a in (a0, a1, a2)]
    dts = np.stack([dot_seq(alt, v).detach().numpy() for v in vp], 1)
    mm = np.zeros(len(p), np.int64)                 # np.argmax: first maximum, NaN wins
    for r in range(len(p)):
        if not np.isnan(dts[r, 0]):
            for k in (1, 2):
                if np.isnan(dts[r, k]):
                    mm[r] = k
                    break
                if dts[r, k] > dts[r, mm[r]]:
                    mm[r] = k
    vpa = torch.stack(vp, 1)
    vtop = vpa[torch.arange(len(p)), torch.as_tensor(mm)]
    south = -alt
    axis = normalize(cross(vtop, south))
    ang, ylat = arc_angle(axis, vtop, south)
    dl = 1.0 / (torch.sqrt(density) * rp)
    nl = torch.as_tensor(count(dl.numpy(), ang.detach().numpy()), dtype=torch.float64)
    cs = (rp * ang) / nl
    fx, fy = circle_frame(south)
    lat = sub_point(torch.zeros_like(south), torch.full_like(ang, rp), vtop, ylat, dl, l)
    dt = dot_seq(lat, south)
    cen = south * dt[:, None]
    rad = torch.sqrt(rp * rp - dt * dt)
    delta = 1.0 / (torch.sqrt(density) * rad)
    nc = torch.as_tensor(count(delta.detach().numpy(), np.full(len(p), TWO_PI)), dtype=torch.float64)
    area = ((rad * TWO_PI) / nc) * cs
    return sub_point(cen, rad, fx, fy, delta, i) + pijk, area


def dots(X, R, dens, rp, topo, m):
    """Positions (n, 3) and areas (n) of molecule m's dots in export order."""
    d = topo["dots"][m]
    n = len(d["type"])
    out_p = torch.zeros((n, 3), dtype=torch.float64)
    out_a = torch.zeros(n, dtype=torch.float64)
    parts = []
    for typ in (1, 2, 3):
        sel = np.nonzero(d["type"] == typ)[0]
        if len(sel) == 0:
            continue
        unit, sub = d["unit"][sel], d["sub"][sel]
        if typ == 1:
            p, a = convex_dots(X, R, topo["dens"], rp, topo["frame"], unit, sub)
        elif typ == 2:
            p, a = toroidal_dots(X, R, topo["dens"], rp, topo["a1"], topo["a2"], unit, sub)
        else:
            p, a = concave_dots(X, R, topo["dens"], rp, topo["pa"], topo["plus"], unit, sub)
        parts.append((torch.as_tensor(sel), p, a))
    for sel, p, a in parts:
        out_p = out_p.index_copy(0, sel, p)
        out_a = out_a.index_copy(0, sel, a)
    return out_p, out_a


def contact_ms(X, R, rp, weight, topo, side=1):
    """sum over the side's buried dots of area * exp(-w d^2), d to the chosen nearest dot."""
    pq, aq = dots(X, R, topo["dens"], rp, topo, side)
    pr, _ = dots(X, R, topo["dens"], rp, topo, 1 - side)
    q = np.nonzero(topo["dots"][side]["bur"])[0]
    r = np.nonzero(topo["dots"][1 - side]["bur"])[0]
    nn = topo["nn"][side]
    diff = pr[torch.as_tensor(r[nn])] - pq[torch.as_tensor(q)]
    d2 = (diff[:, 0] * diff[:, 0] + diff[:, 1] * diff[:, 1]) + diff[:, 2] * diff[:, 2]
    return (aq[torch.as_tensor(q)] * torch.exp(-d2 * weight)).sum()


def topology(ctx, c, density=15.0, nearest=None):
    """
    Export the topology of complex c of a generated context.  nearest(q, r)
    -> (min d2, first argmin) picks each query dot's nearest dot (default:
    scipy cdist; the library's exact search gives the same indices).
    """
    from scipy.spatial.distance import cdist
    info = ctx.info(c)
    n = int(info.n_atoms)
    nb_off, nb_id, _, _ = ctx.export_neighbors(c, n, info)
    frame = np.full(n, -1, np.int64)
    has = nb_off[1:] > nb_off[:-1]
    frame[has] = nb_id[nb_off[:-1][has]]
    a1, a2, _, _, _, _ = ctx.export_toroid(c, info)
    p0, p1, p2, _, _, _ = ctx.export_probes(c, info)
    nplus = int(info.n_probes_plus[0] + info.n_probes_plus[1])
    plus = np.arange(len(p0)) < nplus
    dots_ = []
    for m in (0, 1):
        coor, _, area, bur, typ, atom = ctx.export_dots(c, m, info)
        unit, sub = ctx.export_dot_units(c, m, info)
        dots_.append(dict(coor=coor, area=area, bur=bur.astype(bool), type=typ.astype(np.int64),
                          unit=unit.astype(np.int64), sub=sub.astype(np.int64)))
    nn = []
    for m in (0, 1):
        q = dots_[m]["coor"][dots_[m]["bur"]]
        r = dots_[1 - m]["coor"][dots_[1 - m]["bur"]]
        if not (len(q) and len(r)):
            nn.append(np.zeros(0, np.int64))
        elif nearest is not None:
            nn.append(np.asarray(nearest(q, r)[1], np.int64))
        else:
            nn.append(np.argmin(cdist(r, q, "sqeuclidean"), axis=0))
    return dict(frame=frame, a1=a1.astype(np.int64), a2=a2.astype(np.int64),
                pa=(p0.astype(np.int64), p1.astype(np.int64), p2.astype(np.int64)), plus=plus,
                dots=dots_, nn=nn, dens=np.full(n, float(density)))
