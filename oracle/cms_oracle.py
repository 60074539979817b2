"""
CPU oracle for the contact-molecular-surface (CMS) / shape-complementarity (SC)
pipeline -- TEST INFRASTRUCTURE ONLY.

This module is the checker for the CUDA implementation in ``cms-cuda_b200``.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it; the product path never does.

It is a restatement, in NumPy, of the algorithm of the reference package's
CPU calculator ``cms-cuda/_core.py`` (ullahsamee/cms-cuda, itself the
py_contact_ms port of Longxing Cao's C++ code).  Every floating-point
expression keeps the reference's operation order, written out explicitly so
that the order does not depend on how a NumPy build vectorises a reduction:

* ``dot_seq``  -- ``np.sum(a*b, -1)``, ``np.linalg.norm``, ``scipy cdist``:
  ``(p0 + p1) + p2``;
* ``dot_alt``  -- ``np.einsum('...i,...i')``: ``(p0 + p2) + p1``;
* ``x**2`` is ``x*x``; no fused multiply-add anywhere.

Transcendentals (``sin``, ``cos``, ``arctan2``, ``arccos``, ``exp``) and the
final reductions (``np.bincount``, ``.sum()``, ``.mean()``) are the same NumPy
calls the reference makes, so on the machine that generated the golden
fixtures the oracle reproduces the reference bit for bit (pinned by
``tests/test_oracle.py`` against ``tests/golden``).

Two deliberate differences from the reference, neither of which changes a
result on inputs without exact distance ties:

* neighbour rows are ordered by ``(d2, j)`` with a stable sort; the reference
  uses ``np.argsort`` (unstable) on ``d2`` alone (``_core.py:1331``);
* the all-pairs distance matrices are evaluated in row blocks instead of one
  dense ``(N, N)`` ``cdist`` (``_core.py:1274``), which bounds memory.
"""

import math

import numpy as np

MAX_SUBDIV = 100                 # _core.py:618
ATTEN_BLOCKER = 1                # _core.py:613-616
ATTEN_2 = 2
ATTEN_BURIED_FLAGGED = 5
ATTEN_6 = 6
TWO_PI = 2 * np.pi


# ----------------------------------------------------------------------------
# fixed-order 3-vector arithmetic
# ----------------------------------------------------------------------------

def dot_seq(a, b):
    """np.sum(a * b, axis=-1) / cdist order: (a0*b0 + a1*b1) + a2*b2."""
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def dot_alt(a, b):
    """np.einsum('...i,...i->...') order: (a0*b0 + a2*b2) + a1*b1."""
    return (a[..., 0] * b[..., 0] + a[..., 2] * b[..., 2]) + a[..., 1] * b[..., 1]


def norm(a):
    """np.linalg.norm(a, axis=-1): sqrt of the sequential sum of squares."""
    return np.sqrt(dot_seq(a, a))


def normalize(a):
    """a / np.linalg.norm(a, axis=-1, keepdims=True) (per-component division)."""
    return a / norm(a)[..., None]


def cross(a, b):
    """np.cross for 3-vectors."""
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


# ----------------------------------------------------------------------------
# settings and containers
# ----------------------------------------------------------------------------

class Settings:
    """Defaults of _core.py:766-773."""

    def __init__(self, **kw):
        self.rp = 1.7
        self.density = 15.0
        self.band = 1.5
        self.sep = 8.0
        self.weight = 0.5
        self.binwidth_dist = 0.02
        self.binwidth_norm = 0.02
        for k, v in kw.items():
            setattr(self, k, v)


class CoincidentAtomsError(RuntimeError):
    pass


# ----------------------------------------------------------------------------
# arc / circle subdivision  (_core.py:2380-2527)
# ----------------------------------------------------------------------------

def sub_div(cen, rad, x, y, angle, density):
    """
    vec_sub_div (_core.py:2429-2486), per element: point i exists iff
    delta*(i+0.5) <= angle and i < MAX_SUBDIV, with delta = 1/(sqrt(density)*rad);
    point = (cen + x*(rad*cos a)) + y*(rad*sin a); ps = rad*angle/count.

    Returns (ps (...), points (..., W, 3) NaN-padded, count (...)).
    """
    rad = np.asarray(rad, dtype=np.float64)
    density = np.asarray(density, dtype=np.float64)
    angle = np.asarray(angle, dtype=np.float64)
    base = rad.shape
    with np.errstate(divide='ignore', invalid='ignore', over='ignore'):
        delta = 1.0 / (np.sqrt(density) * rad)
        raw = angle / delta
    ok = np.isfinite(raw) & (raw > 0)
    if not ok.any():
        return np.zeros(base), np.full(base + (0, 3), np.nan), np.zeros(base, dtype=np.int64)
    width = int(min(MAX_SUBDIV, math.ceil(float(raw[ok].max()))))
    if width == 0:
        return np.zeros(base), np.full(base + (0, 3), np.nan), np.zeros(base, dtype=np.int64)
    i = np.arange(width)
    with np.errstate(invalid='ignore', over='ignore'):
        a = delta[..., None] * (i + 0.5)
        mask = a <= angle[..., None]
        c = rad[..., None] * np.cos(a)
        s = rad[..., None] * np.sin(a)
        pts = (cen[..., None, :] + x[..., None, :] * c[..., None]) + y[..., None, :] * s[..., None]
    pts = np.where(mask[..., None], pts, np.nan)
    count = mask.sum(axis=-1)
    with np.errstate(invalid='ignore', divide='ignore'):
        ps = np.where(count > 0, (rad * angle) / np.maximum(count, 1).astype(np.float64), 0.0)
    return ps, pts, count


def sub_arc(cen, rad, axis, density, x, v):
    """vec_sub_arc (_core.py:2407-2427)."""
    y = cross(axis, x)
    dt1 = dot_seq(v, x)
    dt2 = dot_seq(v, y)
    angle = np.arctan2(dt2, dt1)
    angle = np.where(angle < 0.0, angle + TWO_PI, angle)
    angle = np.where((np.abs(dt1) <= 1e-08) & (np.abs(dt2) <= 1e-08), np.nan, angle)
    return sub_div(cen, rad, x, y, angle, density)


def circle_frame(axis):
    """The (x, y) in-plane frame of vec_sub_cir (_core.py:2488-2523)."""
    axis = normalize(axis)
    v1 = np.stack([axis[..., 1] * axis[..., 1] + axis[..., 2] * axis[..., 2],
                   axis[..., 0] * axis[..., 0] + axis[..., 2] * axis[..., 2],
                   axis[..., 0] * axis[..., 0] + axis[..., 1] * axis[..., 1]], axis=-1)
    v1 = normalize(v1)
    dt = dot_seq(v1, axis)
    v1 = np.where((np.abs(dt) > 0.99)[..., None], np.array([1.0, 0.0, 0.0]), v1)
    v2 = normalize(cross(axis, v1))
    x = normalize(cross(axis, v2))
    y = cross(axis, x)
    return x, y


def sub_cir(cen, rad, axis, density):
    """vec_sub_cir (_core.py:2488-2527): full circle, angle 2*pi."""
    x, y = circle_frame(axis)
    angle = np.full(np.shape(rad), TWO_PI)
    return sub_div(cen, rad, x, y, angle, density)


def distance_point_to_line(cen, axis, pnt):
    """vec_distance_point_to_line (_core.py:2380-2386)."""
    vec = pnt - cen
    dt = dot_seq(vec, axis)
    d2 = dot_seq(vec, vec) - dt * dt
    with np.errstate(invalid='ignore'):
        return np.where(d2 < 0.0, 0.0, np.sqrt(np.where(d2 < 0.0, 0.0, d2)))


# ----------------------------------------------------------------------------
# the surface calculation of one complex
# ----------------------------------------------------------------------------

class Surface:
    """
    Everything the reference keeps in ``calc.run`` after surface generation.

    Atom arrays are indexed by natom (binder atoms first, then target atoms,
    _core.py:372-399).  Neighbour tables are CSR lists here (row i of the
    reference's padded SimpleNeighborArray is nb_id[nb_off[i]:nb_off[i+1]]).
    """


def _blocks(n, rows=2048):
    for s in range(0, n, rows):
        yield s, min(n, s + rows)


def build_surface(xyz, radius, molecule, density, settings, all_atoms=False):
    """
    _ensure_surfaces_generated (_core.py:865-909): attention numbers, neighbour
    lists, pair and triple loops, then convex, toroidal and concave dots.
    """
    st = settings
    rp = float(st.rp)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    radius = np.ascontiguousarray(radius, dtype=np.float64)
    molecule = np.ascontiguousarray(molecule, dtype=np.int8)
    density = np.broadcast_to(np.asarray(density, dtype=np.float64), radius.shape).copy()
    N = len(radius)
    assert N > 0
    S = Surface()
    S.settings = st
    S.all_atoms = bool(all_atoms)
    S.xyz, S.radius, S.molecule, S.density = xyz, radius, molecule, density
    S.natom = np.arange(N, dtype=np.int32)
    S.access = np.zeros(N, dtype=np.int8)
    S.counts = dict(convex=0, toroidal=0, concave=0)
    S.n_blocked = [0, 0]
    S.n_buried_atoms = [0, 0]

    # ---- attention numbers (_core.py:1150-1195) -----------------------------
    atten = np.zeros(N, dtype=np.int8)
    if all_atoms:
        atten[:] = ATTEN_BURIED_FLAGGED
        for m in range(2):
            S.n_buried_atoms[m] += int((molecule == m).sum())
    else:
        i0 = np.where(molecule == 0)[0]
        i1 = np.where(molecule == 1)[0]
        min0 = np.full(len(i0), np.inf)
        min1 = np.full(len(i1), np.inf)
        if len(i0) and len(i1):
            for s, e in _blocks(len(i0)):
                d = xyz[i0[s:e], None, :] - xyz[None, i1, :]
                d2 = dot_seq(d, d)
                min0[s:e] = d2.min(axis=1)
                min1 = np.minimum(min1, d2.min(axis=0))
            # cdist(xyz0, xyz1) is sqrt of the cdist-order squared distance;
            # sqrt is monotone and correctly rounded, so min commutes with it
            min0 = np.sqrt(min0)
            min1 = np.sqrt(min1)
        else:
            min0[:] = 99999.0
            min1[:] = 99999.0
        b0 = min0 >= st.sep
        b1 = min1 >= st.sep
        atten[i0[b0]] = ATTEN_BLOCKER
        atten[i0[~b0]] = ATTEN_BURIED_FLAGGED
        atten[i1[b1]] = ATTEN_BLOCKER
        atten[i1[~b1]] = ATTEN_BURIED_FLAGGED
        S.n_blocked[0] += int(b0.sum()); S.n_buried_atoms[0] += int((~b0).sum())
        S.n_blocked[1] += int(b1.sum()); S.n_buried_atoms[1] += int((~b1).sum())
    S.atten = atten
    S.radmax = float(radius.max())

    # ---- neighbour and buried-partner lists (_core.py:1251-1349) ------------
    active = atten > 0
    nb_rows, bu_rows = [None] * N, [None] * N
    nn = np.zeros(N, dtype=np.int32)
    nbur = np.zeros(N, dtype=np.int32)
    coincident = None
    for s, e in _blocks(N, 1024):
        d = xyz[s:e, None, :] - xyz[None, :, :]
        d2 = dot_seq(d, d)                                        # cdist sqeuclidean
        r_sum = radius[s:e, None] + radius[None, :]
        bridge2 = (r_sum + 2.0 * rp) * (r_sum + 2.0 * rp)
        same = molecule[s:e, None] == molecule[None, :]
        off = same.copy()
        off[np.arange(e - s), np.arange(s, e)] = False
        act2 = active[s:e, None] & active[None, :]
        coin = off & act2 & (d2 <= 0.0001)
        if coincident is None and coin.any():
            r0, c0 = np.argwhere(coin)[0]
            coincident = (s + int(r0), int(c0))
        nmask = act2 & off & (d2 < bridge2)
        bmask = active[s:e, None] & (atten >= ATTEN_BURIED_FLAGGED)[None, :] & ~same & (d2 < bridge2)
        for r in range(e - s):
            i = s + r
            j = np.where(nmask[r])[0]
            if len(j):
                j = j[np.lexsort((j, d2[r, j]))]                   # by (d2, j)
            nb_rows[i] = j.astype(np.int32)
            nn[i] = len(j)
            jb = np.where(bmask[r])[0]
            bu_rows[i] = jb.astype(np.int32)
            nbur[i] = len(jb)
    if coincident is not None:
        i0_, j0_ = coincident
        raise CoincidentAtomsError(f"Coincident atoms: {i0_}:: == {j0_}::")
    S.nb_off = np.concatenate([[0], np.cumsum(nn)]).astype(np.int64)
    S.nb_id = np.concatenate(nb_rows).astype(np.int32) if N else np.zeros(0, np.int32)
    S.bu_off = np.concatenate([[0], np.cumsum(nbur)]).astype(np.int64)
    S.bu_id = np.concatenate(bu_rows).astype(np.int32) if N else np.zeros(0, np.int32)
    S.nn, S.nbur = nn, nbur
    # atten6_no_nbb is always False: ATTEN_6 is never assigned (_core.py:1311)
    S.access |= (active & (nn == 0)).astype(np.int8)
    good = active & (nn > 0)
    S.max_nn = max(int(nn.max()) if nn.any() else 1, 1)
    S.max_nbur = max(int(nbur.max()) if nbur.any() else 1, 1)

    # padded (N, K) neighbour views, the layout of SimpleNeighborArray
    K = S.max_nn
    pad_id = np.full((N, K), -1, dtype=np.int32)
    for i in range(N):
        pad_id[i, :nn[i]] = S.nb_id[S.nb_off[i]:S.nb_off[i + 1]]
    S.pad_id = pad_id
    safe = np.where(pad_id >= 0, pad_id, 0)
    S.pad_xyz = np.where((pad_id >= 0)[..., None], xyz[safe], np.nan)
    S.pad_rad = np.where(pad_id >= 0, radius[safe], np.nan)
    KB = S.max_nbur
    bpad = np.full((N, KB), -1, dtype=np.int32)
    for i in range(N):
        bpad[i, :nbur[i]] = S.bu_id[S.bu_off[i]:S.bu_off[i + 1]]
    S.bpad_id = bpad
    bsafe = np.where(bpad >= 0, bpad, 0)
    S.bpad_xyz = np.where((bpad >= 0)[..., None], xyz[bsafe], np.nan)
    S.bpad_rad = np.where(bpad >= 0, radius[bsafe], np.nan)

    S.dots = [[], []]          # per molecule: list of dict batches, in add_dots call order
    S.toroid = None
    S.probes = None

    good_idx = np.where(good)[0]
    _pair_and_triple_loops(S, good_idx)

    # ---- convex queue (_core.py:1212-1222) ----------------------------------
    conv = good_idx[(S.access[good_idx] != 0) & (atten[good_idx] > ATTEN_BLOCKER)]
    _convex(S, conv)
    _toroidal(S)
    if rp > 0:
        _concave(S)
    S.dot_arrays = [_concat_dots(S.dots[m]) for m in (0, 1)]
    return S


def _pair_and_triple_loops(S, good_idx):
    """second_loop (_core.py:1351-1442) and vec_third_loop (_core.py:1445-1643)."""
    rp = float(S.settings.rp)
    xyz, radius, atten = S.xyz, S.radius, S.atten
    empty_tq = dict(i=np.zeros(0, np.int32), j=np.zeros(0, np.int32), uij=np.zeros((0, 3)),
                    tij=np.zeros((0, 3)), rij=np.zeros(0), between=np.zeros(0, bool))
    S.toroid = empty_tq
    S.probes = dict(a0=np.zeros(0, np.int32), a1=np.zeros(0, np.int32), a2=np.zeros(0, np.int32),
                    height=np.zeros(0), point=np.zeros((0, 3)), alt=np.zeros((0, 3)))
    if len(good_idx) == 0:
        return
    na1 = good_idx
    nneigh = S.nn[na1]
    nxyz = S.pad_xyz[na1]
    nrad = S.pad_rad[na1]
    nid = S.pad_id[na1]
    fwd = nid > na1[:, None]
    ax = xyz[na1]
    diff = nxyz - ax[:, None, :]
    dij_sq = dot_alt(diff, diff)
    with np.errstate(invalid='ignore', divide='ignore'):
        dij = np.sqrt(np.where(fwd, dij_sq, 1.0))
        eri = radius[na1] + rp
        erj = nrad + rp
        asymm = np.where(fwd, (eri[:, None] * eri[:, None] - erj * erj) / dij, 0.0)
        between = np.abs(asymm) < dij
        tij = ((ax[:, None, :] + nxyz) * 0.5) + (diff / dij[..., None]) * (asymm * 0.5)[..., None]
        far_sq = np.where(fwd, (eri[:, None] + erj) * (eri[:, None] + erj) - dij_sq, -1.0)
        rdiff = radius[na1][:, None] - nrad
        cont_sq = np.where(fwd, dij_sq - rdiff * rdiff, -1.0)
    geom_ok = fwd & (far_sq > 0.0) & (cont_sq > 0.0)

    shortcut = (nneigh <= 1) & geom_ok.any(axis=1)
    if shortcut.any():
        S.access[na1[shortcut]] = 1
        first_k = np.argmax(geom_ok[shortcut], axis=1)
        S.access[nid[shortcut][np.arange(int(shortcut.sum())), first_k]] = 1

    pair_mask = geom_ok & ~shortcut[:, None]
    pi_, pk_ = np.where(pair_mask)
    if len(pi_) == 0:
        return
    p_i = na1[pi_].astype(np.int32)
    p_j = nid[pi_, pk_].astype(np.int32)
    p_dij = dij[pi_, pk_]
    p_uij = diff[pi_, pk_] / p_dij[:, None]
    p_tij = tij[pi_, pk_]
    p_rij = ((0.5 * np.sqrt(far_sq[pi_, pk_])) * np.sqrt(cont_sq[pi_, pk_])) / p_dij
    p_bet = between[pi_, pk_]
    need_tor = (atten[p_i] > ATTEN_BLOCKER) | ((atten[p_j] > ATTEN_BLOCKER) & (rp > 0.0))
    S.toroid = dict(i=p_i[need_tor], j=p_j[need_tor], uij=p_uij[need_tor], tij=p_tij[need_tor],
                    rij=p_rij[need_tor], between=p_bet[need_tor])
    S.pairs = dict(i=p_i, j=p_j)

    # ---- triples ------------------------------------------------------------
    M = len(p_i)
    eri = radius[p_i] + rp
    erj = radius[p_j] + rp
    txyz = S.pad_xyz[p_i]
    trad = S.pad_rad[p_i]
    tid = S.pad_id[p_i]
    valid = (tid > p_j[:, None]) & (tid >= 0)
    with np.errstate(invalid='ignore'):
        erk = np.where(valid, trad + rp, np.inf)
        djk = norm(txyz - xyz[p_j][:, None, :])
        valid &= djk < (erj[:, None] + erk)
        dik = norm(txyz - xyz[p_i][:, None, :])
        valid &= dik < (eri[:, None] + erk)
    a3 = atten[np.where(tid >= 0, tid, 0)]
    all_blocked = ((atten[p_i][:, None] <= ATTEN_BLOCKER) & (atten[p_j][:, None] <= ATTEN_BLOCKER)
                   & (a3 <= ATTEN_BLOCKER))
    valid &= ~all_blocked
    if not valid.any():
        return
    q_p, q_k = np.where(valid)
    x1 = xyz[p_i[q_p]]
    x3 = txyz[q_p, q_k]
    n3 = tid[q_p, q_k]
    erk_q = trad[q_p, q_k] + rp
    eri_q = eri[q_p]
    dik_q = dik[q_p, q_k]
    uij_q = p_uij[q_p]
    tij_q = p_tij[q_p]
    rij_q = p_rij[q_p]
    uik = (x3 - x1) / dik_q[:, None]
    dt = dot_alt(uij_q, uik)
    wijk = np.arccos(np.clip(dt, -1.0, 1.0))
    swijk = np.sin(wijk)
    degenerate = (dt >= 1.0) | (dt <= -1.0) | (wijk <= 0.0) | (swijk <= 0.0)
    keep = ~degenerate
    if degenerate.any():
        dd = tij_q - x3
        dtijk2 = dot_seq(dd, dd)
        rkp2 = erk_q * erk_q - rij_q * rij_q
        kills = degenerate & (dtijk2 < rkp2)
        if kills.any():
            killed = np.zeros(M, dtype=bool)
            killed[q_p[kills]] = True
            keep &= ~killed[q_p]
    if not keep.any():
        return
    q_p, n3 = q_p[keep], n3[keep]
    x1, x3 = x1[keep], x3[keep]
    eri_q, erk_q, dik_q = eri_q[keep], erk_q[keep], dik_q[keep]
    uij_q, tij_q, uik, swijk = uij_q[keep], tij_q[keep], uik[keep], swijk[keep]
    uijk = cross(uij_q, uik) / swijk[:, None]
    utb = cross(uijk, uij_q)
    asymm_q = (eri_q * eri_q - erk_q * erk_q) / dik_q
    tik = (x1 + x3) * 0.5 + uik * (asymm_q * 0.5)[:, None]
    dt_b = dot_alt(uik, tik - tij_q)
    bijk = tij_q + utb * (dt_b / swijk)[:, None]
    bma = bijk - x1
    h2 = eri_q * eri_q - dot_alt(bma, bma)
    vh = h2 > 0.0
    if not vh.any():
        return
    bijk, uijk, h = bijk[vh], uijk[vh], np.sqrt(h2[vh])
    q_p, n3 = q_p[vh], n3[vh]
    n1, n2 = p_i[q_p], p_j[q_p]
    Q = len(h)
    sign = np.concatenate([np.ones(Q), -np.ones(Q)])
    b2 = np.concatenate([bijk, bijk])
    u2 = np.concatenate([uijk, uijk])
    h2q = np.concatenate([h, h])
    pijk = b2 + u2 * (h2q * sign)[:, None]
    alt = u2 * sign[:, None]
    n1_2, n2_2, n3_2 = np.concatenate([n1, n1]), np.concatenate([n2, n2]), np.concatenate([n3, n3])
    a0 = np.where(sign > 0, n1_2, n2_2)
    a1 = np.where(sign > 0, n2_2, n1_2)
    # collision against atom1's neighbours except atom2 and atom3 (alt order, <=)
    cx, cr, cid = S.pad_xyz[n1_2], S.pad_rad[n1_2], S.pad_id[n1_2]
    excl = (cid == n2_2[:, None]) | (cid == n3_2[:, None]) | (cid < 0)
    rows, cols = np.where(~excl)
    dd = pijk[rows] - cx[rows, cols]
    hit = dot_alt(dd, dd) <= (cr[rows, cols] + rp) * (cr[rows, cols] + rp)
    coll = np.zeros(len(pijk), dtype=bool)
    coll[rows[hit]] = True
    ok = ~coll
    if not ok.any():
        return
    S.probes = dict(a0=a0[ok].astype(np.int32), a1=a1[ok].astype(np.int32), a2=n3_2[ok].astype(np.int32),
                    height=h2q[ok], point=pijk[ok], alt=alt[ok])
    acc = np.unique(np.concatenate([S.probes['a0'], S.probes['a1'], S.probes['a2']]))
    S.access[acc] = 1


def _add_dots(S, molecule, type_, coor, area, pcen, owner):
    """add_dots (_core.py:2337-2377): outward normal, burial test, per-molecule append."""
    n = len(coor)
    if n == 0:
        return
    rp = float(S.settings.rp)
    owner = np.asarray(owner, dtype=np.int32)
    molecule = np.asarray(molecule, dtype=np.int8)
    if rp <= 0:
        nml = coor - S.xyz[owner]
    else:
        nml = (pcen - coor) / rp
    bx = S.bpad_xyz[owner]
    br = S.bpad_rad[owner]
    d = bx - pcen[:, None, :]
    with np.errstate(invalid='ignore'):
        buried = (dot_seq(d, d) <= (br + rp) * (br + rp)).any(axis=-1).astype(np.int8)
    for m in (0, 1):
        sel = molecule == m
        if sel.any():
            S.dots[m].append(dict(coor=coor[sel], nml=nml[sel], area=area[sel], buried=buried[sel],
                                  type=np.full(int(sel.sum()), type_, np.int8), atom=owner[sel]))


def _concat_dots(batches):
    if not batches:
        return dict(coor=np.zeros((0, 3)), nml=np.zeros((0, 3)), area=np.zeros(0),
                    buried=np.zeros(0, np.int8), type=np.zeros(0, np.int8), atom=np.zeros(0, np.int32))
    return {k: np.concatenate([b[k] for b in batches]) for k in batches[0]}


def _circle_points(cen, rad, axis, density):
    """Subdivide every (row, latitude) circle with rad > 0 (the tail of convex/concave)."""
    R, M = rad.shape
    flat = rad.reshape(-1)
    act = flat > 0
    if act.any():
        ps_a, pts_a, _ = sub_cir(cen.reshape(-1, 3)[act], flat[act],
                                 np.repeat(axis, M, axis=0)[act], np.repeat(density, M)[act])
        W = pts_a.shape[1]
        pts = np.full((R * M, W, 3), np.nan)
        pts[act] = pts_a
        ps = np.zeros(R * M)
        ps[act] = ps_a
    else:
        W = 0
        pts = np.empty((R * M, 0, 3))
        ps = np.zeros(R * M)
    return pts.reshape(R, M, W, 3), ps.reshape(R, M)


def _convex(S, q):
    """generate_convex_surface + vec_check_point_collision (_core.py:1646-1840)."""
    N = len(q)
    if N == 0:
        return
    rp = float(S.settings.rp)
    axyz = S.xyz[q]
    ri = S.radius[q]
    eri = ri + rp
    dens = S.density[q]
    north = np.tile([0.0, 0.0, 1.0], (N, 1))
    south = np.tile([0.0, 0.0, -1.0], (N, 1))
    eqvec = np.tile([1.0, 0.0, 0.0], (N, 1))
    has = S.nn[q] > 0
    if has.any():
        nx = S.pad_xyz[q, 0]
        nr = S.pad_rad[q, 0]
        with np.errstate(invalid='ignore', divide='ignore'):
            north[has] = normalize(axyz - nx)[has]
            vt = np.stack([north[:, 1] * north[:, 1] + north[:, 2] * north[:, 2],
                           north[:, 0] * north[:, 0] + north[:, 2] * north[:, 2],
                           north[:, 0] * north[:, 0] + north[:, 1] * north[:, 1]], axis=-1)
            vt = normalize(vt)
            dt = dot_seq(vt, north)
            vt[np.abs(dt) > 0.99] = np.array([1.0, 0.0, 0.0])
            eq = normalize(cross(north, vt))
            eqvec[has] = eq[has]
            vql = cross(eqvec, north)
            erj = nr + rp
            dij = norm(nx - axyz)
            uij = (nx - axyz) / dij[:, None]
            asymm = (eri * eri - erj * erj) / dij
            tij = ((axyz + nx) * 0.5) + uij * (asymm[:, None] * 0.5)
            far_sq = (eri + erj) * (eri + erj) - dij * dij
            rd = ri - nr
            contain_sq = dij * dij - rd * rd
            geom_ok = has & (far_sq > 0.0) & (contain_sq > 0.0)
            far = np.sqrt(np.where(geom_ok, far_sq, 1.0))
            contain = np.sqrt(np.where(geom_ok, contain_sq, 1.0))
            rij = ((0.5 * far) * contain) / dij
            pij = tij + vql * rij[:, None]
            south_vec = (pij - axyz) / eri[:, None]
        south[geom_ok] = south_vec[geom_ok]
    cs, lats, _ = sub_arc(np.zeros((N, 3)), ri, eqvec, dens, north, south)
    with np.errstate(invalid='ignore'):
        dt = dot_seq(lats, north[:, None, :])
        cen = axyz[:, None, :] + dt[..., None] * north[:, None, :]
        rad_sq = ri[:, None] * ri[:, None] - dt * dt
    rad = np.zeros_like(rad_sq)
    vr = rad_sq > 0
    rad[vr] = np.sqrt(rad_sq[vr])
    pts, ps = _circle_points(cen, rad, north, dens)
    area = ps * cs[:, None]
    valid = ~np.isnan(pts[..., 0])
    a_i, l_i, _ = np.where(valid)
    pflat = pts[valid]
    with np.errstate(invalid='ignore', divide='ignore'):
        pcen = axyz[a_i] + (pflat - axyz[a_i]) * (eri[a_i] / ri[a_i])[:, None]
    # collision with every neighbour except slot 0 (seq order, <=)
    nb = S.pad_xyz[q][a_i]
    nbr = S.pad_rad[q][a_i]
    d = nb - pcen[:, None, :]
    with np.errstate(invalid='ignore'):
        hit = (dot_seq(d, d) <= (nbr + rp) * (nbr + rp)) & ~np.isnan(nbr)
    coll = hit[:, 1:].any(axis=-1)
    keep = ~coll
    if not keep.any():
        return
    S.counts['convex'] += int(keep.sum())
    ak = a_i[keep]
    _add_dots(S, S.molecule[q][ak], 1, pflat[keep], area[ak, l_i[keep]], pcen[keep], q[ak])


def _toroidal(S):
    """generate_toroidal_surface(s) (_core.py:1234-1248, 1847-2067)."""
    T = S.toroid
    n1, n2 = T['i'], T['j']
    N = len(n1)
    S.tor_access1 = np.zeros(N, dtype=bool)
    S.tor_access2 = np.zeros(N, dtype=bool)
    if N == 0:
        _apply_tor_access(S)
        return
    rp = float(S.settings.rp)
    uij, tij, rij, between = T['uij'], T['tij'], T['rij'], T['between']
    r1, r2 = S.radius[n1], S.radius[n2]
    density = (S.density[n1] + S.density[n2]) * 0.5
    eri, erj = r1 + rp, r2 + rp
    with np.errstate(invalid='ignore', divide='ignore'):
        rci = (rij * r1) / eri
        rcj = (rij * r2) / erj
        rb = np.maximum(rij - rp, 0.0)
        rs = ((rci + 2 * rb) + rcj) * 0.25
        e = rs / rij
        edens = (e * e) * density
    ts, subs, _ = sub_cir(tij, rij, uij, edens)
    vsub = ~np.isnan(subs[..., 0])
    if not vsub.any():
        _apply_tor_access(S)
        return
    p_idx, _ = np.where(vsub)
    pij = subs[vsub]
    cx, cr, cid = S.pad_xyz[n1][p_idx], S.pad_rad[n1][p_idx], S.pad_id[n1][p_idx]
    excl = (cid < 0) | (cid == n2[p_idx, None])
    rows, cols = np.where(~excl)
    dd = pij[rows] - cx[rows, cols]
    hit = dot_alt(dd, dd) < (cr[rows, cols] + rp) * (cr[rows, cols] + rp)
    close = np.zeros(len(pij), dtype=bool)
    close[rows[hit]] = True
    ok = ~close
    if not ok.any():
        _apply_tor_access(S)
        return
    pij, p_idx = pij[ok], p_idx[ok]
    S.tor_access1[p_idx] = True
    S.tor_access2[p_idx] = True
    with np.errstate(invalid='ignore', divide='ignore'):
        pi = (S.xyz[n1][p_idx] - pij) / eri[p_idx, None]
        pj = (S.xyz[n2][p_idx] - pij) / erj[p_idx, None]
        axis = normalize(cross(pi, pj))
        rr = rij[p_idx]
        dtq = rp * rp - rr * rr
        cusp = (dtq > 0) & between[p_idx]
        dtq_s = np.sqrt(np.where(cusp, dtq, 0.0))
        qij = tij[p_idx] - uij[p_idx] * dtq_s[:, None]
        pqi_c = (qij - pij) / rp
        mid = normalize(pi + pj)
    pqi = np.where(cusp[:, None], pqi_c, mid)
    pqj = np.where(cusp[:, None], 0.0, mid)
    dt1 = dot_seq(pqi, pi)
    dt2 = dot_seq(pqj, pj)
    va = (np.abs(dt1) < 1.0) & (np.abs(dt2) < 1.0)
    if not va.any():
        _apply_tor_access(S)
        return
    pij, axis, pi, pj, pqi, pqj, p_idx = pij[va], axis[va], pi[va], pj[va], pqi[va], pqj[va], p_idx[va]
    mol1 = S.molecule[n1][p_idx]
    for arc in (1, 2):
        m = (S.atten[n1][p_idx] if arc == 1 else S.atten[n2][p_idx]) >= ATTEN_2
        if not m.any():
            continue
        pid = p_idx[m]
        x, v = (pi[m], pqi[m]) if arc == 1 else (pqj[m], pj[m])
        ps, pts, _ = sub_arc(pij[m], np.full(int(m.sum()), rp), axis[m], density[pid], x, v)
        with np.errstate(invalid='ignore', divide='ignore'):
            dist = distance_point_to_line(tij[pid][:, None, :], uij[pid][:, None, :], pts)
            areas = ((ps[:, None] * ts[pid, None]) * dist) / rij[pid, None]
        valid = ~np.isnan(areas)
        k = int(valid.sum())
        S.counts['toroidal'] += k
        if k:
            owner = (n1 if arc == 1 else n2)[pid]
            mol = np.broadcast_to(mol1[m][:, None], valid.shape)[valid]
            own = np.broadcast_to(owner[:, None], valid.shape)[valid]
            pc = np.broadcast_to(pij[m][:, None, :], pts.shape)[valid]
            _add_dots(S, mol, 2, pts[valid], areas[valid], pc, own)
    _apply_tor_access(S)


def _apply_tor_access(S):
    """
    access[natoms1] |= has1, then access[natoms2] |= has2 (_core.py:1247-1248):
    NumPy fancy-index read-modify-write, so for a repeated index the value
    computed for its last occurrence is the one that remains.
    """
    T = S.toroid
    for idx, has in ((T['i'], S.tor_access1), (T['j'], S.tor_access2)):
        if len(idx) == 0:
            continue
        S.access[idx] |= has.astype(np.int8)


def _concave(S):
    """generate_concave_surface + check_probe_collision_vectorized (_core.py:2069-2333)."""
    P_ = S.probes
    P = len(P_['height'])
    if P == 0:
        return
    rp = float(S.settings.rp)
    rp2 = rp * rp
    pijk, uijk, hijk = P_['point'], P_['alt'], P_['height']
    ids = np.stack([P_['a0'], P_['a1'], P_['a2']], axis=1)
    axyz = S.xyz[ids]                      # (P, 3, 3)
    arad = S.radius[ids]
    adens = S.density[ids]
    amol = S.molecule[ids]
    density = ((adens[:, 0] + adens[:, 1]) + adens[:, 2]) / 3
    low = hijk < rp
    low_pts = pijk[low]
    # probes whose three atoms are all ATTEN_6 are skipped: never true (ATTEN_6 unused)
    nears = None
    if low.any():
        d = pijk[:, None, :] - low_pts[None, :, :]
        nears = dot_seq(d, d) <= 4 * rp2
        li = np.where(low)[0]
        nears[li, np.arange(len(li))] = False
    vp = normalize(axyz - pijk[:, None, :])
    vecs = normalize(np.stack([cross(vp[:, 0], vp[:, 1]), cross(vp[:, 1], vp[:, 2]),
                               cross(vp[:, 2], vp[:, 0])], axis=1))
    dt = dot_seq(uijk[:, None, :], vp)
    mm = np.argmax(dt, axis=1)
    south = -uijk
    vtop = vp[np.arange(P), mm]
    axis = normalize(cross(vtop, south))
    cs, lats, _ = sub_arc(np.zeros_like(pijk), np.full(P, rp), axis, density, vtop, south)
    with np.errstate(invalid='ignore'):
        dtl = dot_seq(lats, south[:, None, :])
        cen = south[:, None, :] * dtl[..., None]
        rad_sq = rp2 - dtl * dtl
        rad = np.sqrt(np.where(rad_sq < 0, 0.0, rad_sq))
    pts, ps = _circle_points(cen, rad, south, density)
    area = ps * cs[:, None]
    valid = ~np.isnan(pts[..., 0])
    ip, il, _ = np.where(valid)
    pt = pts[valid]
    bail = (dot_seq(pt[:, None, :], vecs[ip]) >= 0).any(axis=1)
    pt, ip, il = pt[~bail], ip[~bail], il[~bail]
    pt = pt + pijk[ip]
    if nears is not None:
        sel = nears[ip]
        near_any = sel.any(axis=1)
        rows, cols = np.where(sel)
        dd = pt[rows] - low_pts[cols]
        hit = dot_alt(dd, dd) < rp2
        coll = np.zeros(len(pt), dtype=bool)
        coll[rows[hit]] = True
        rej = (hijk[ip] < rp) & near_any & coll
        pt, ip, il = pt[~rej], ip[~rej], il[~rej]
    dd = norm(pt[:, None, :] - axyz[ip]) - arad[ip]
    mc = np.argmin(dd, axis=1)
    S.counts['concave'] += len(pt)
    _add_dots(S, amol[ip, mc], 3, pt, area[ip, il], pijk[ip], ids[ip, mc])


# ----------------------------------------------------------------------------
# readouts  (_core.py:946-1147)
# ----------------------------------------------------------------------------

def _min_sqdist(q, r, rows=4096):
    """
    cdist(r, q, 'sqeuclidean').min(axis=0) and .argmin(axis=0) (first index on
    ties), evaluated in blocks of reference rows.  SciPy's sqeuclidean kernel
    accumulates (d0*d0 + d1*d1) + d2*d2, the dot_seq order.
    """
    from scipy.spatial.distance import cdist
    best = np.full(len(q), np.inf)
    arg = np.zeros(len(q), dtype=np.int64)
    for s, e in _blocks(len(r), rows):
        d2 = cdist(r[s:e], q, metric='sqeuclidean')
        a = d2.argmin(axis=0)
        v = d2[a, np.arange(len(q))]
        better = v < best
        best = np.where(better, v, best)
        arg = np.where(better, a + s, arg)
    return best, arg


def contact_ms(S, target_side=True):
    """calc_contact_molecular_surface (_core.py:946-1004)."""
    mol = S.molecule
    n1 = int((mol == 1).sum())
    n0 = len(mol) - n1
    if target_side:
        q, r, nq, off = S.dot_arrays[1], S.dot_arrays[0], n1, n0
    else:
        q, r, nq, off = S.dot_arrays[0], S.dot_arrays[1], n0, 0
    zero = (0.0, np.zeros(nq))
    if len(r['area']) == 0:
        return zero
    bq, br = q['buried'].astype(bool), r['buried'].astype(bool)
    if not bq.any() or not br.any():
        return zero
    m2, _ = _min_sqdist(q['coor'][bq], r['coor'][br])
    per_dot = q['area'][bq] * np.exp(-m2 * S.settings.weight)
    per_atom = np.bincount(q['atom'][bq] - off, weights=per_dot, minlength=nq).astype(np.float64)
    return float(per_atom.sum()), per_atom


def max_contact_ms(S):
    """calc_max_possible_contact_molecular_surface (_core.py:1007-1034)."""
    n0 = int((S.molecule == 0).sum())
    d = S.dot_arrays[0]
    if len(d['area']) == 0:
        return 0.0, np.zeros(n0)
    per_atom = np.bincount(d['atom'], weights=d['area'], minlength=n0).astype(np.float64)
    return float(per_atom.sum()), per_atom


def binned_median(values, binwidth):
    """_binned_median (_core.py:1080-1104): grouped-data median."""
    n = len(values)
    if n == 0:
        return 0.0
    ibin = np.floor(values / binwidth).astype(np.int64)
    bins, counts = np.unique(ibin, return_counts=True)
    pct = 100.0 / n
    cum = np.cumsum(counts) * pct
    before = cum - counts * pct
    j = min(int(np.searchsorted(cum, 50.0, side='left')), len(bins) - 1)
    return float(bins[j] * binwidth + (50.0 - before[j]) * binwidth / (counts[j] * pct))


def _trim(S, d):
    """trim_peripheral_band_vectorized (_core.py:1037-1077)."""
    n = len(d['area'])
    bur = d['buried'].astype(bool)
    if not bur.any():
        return 0.0, np.zeros(n, dtype=bool)
    acc = ~bur
    if not acc.any():
        keep = bur.copy()
    else:
        m2, _ = _min_sqdist(d['coor'][bur], d['coor'][acc])
        keep = np.zeros(n, dtype=bool)
        keep[np.where(bur)[0][m2 > S.settings.band ** 2]] = True
    return float(d['area'][keep].sum()), keep


def _neighbor_distance(S, my, their):
    """calc_neighbor_distance_vectorized (_core.py:1107-1147); None if skipped."""
    if len(my['area']) == 0 or len(their['area']) == 0:
        return None
    tb = their['buried'].astype(bool)
    if not tb.any():
        return None
    m2, nn = _min_sqdist(my['coor'], their['coor'][tb])
    distmin = np.sqrt(m2)
    r = dot_alt(my['nml'], their['nml'][tb][nn])
    r = r * np.exp(-(distmin * distmin) * S.settings.weight)
    r = np.clip(r, -0.999, 0.999)
    st = S.settings
    return dict(d_mean=float(distmin.mean()), d_median=binned_median(distmin, st.binwidth_dist),
                s_mean=float(-r.mean()), s_median=float(-binned_median(r, st.binwidth_norm)),
                nn=nn, distmin=distmin, r=r)


def shape_complementarity(S):
    """CalcLoadedSC (_core.py:807-863).  Returns (sc, area, distance, details)."""
    surf = [dict(d_mean=0.0, d_median=0.0, s_mean=0.0, s_median=0.0, trimmedArea=0.0,
                 nTrimmedDots=0, nAllDots=0) for _ in range(3)]
    trimmed = []
    for m in (0, 1):
        d = S.dot_arrays[m]
        area, keep = _trim(S, d)
        trimmed.append({k: v[keep] for k, v in d.items()})
        surf[m].update(trimmedArea=area, nTrimmedDots=int(keep.sum()), nAllDots=len(d['area']))
    extra = []
    for m in (0, 1):
        res = _neighbor_distance(S, trimmed[m], trimmed[1 - m])
        extra.append(res)
        if res is not None:
            for k in ('d_mean', 'd_median', 's_mean', 's_median'):
                surf[m][k] = res[k]
    s0, s1, s2 = surf
    for k in ('d_mean', 'd_median', 's_mean', 's_median'):
        s2[k] = (s0[k] + s1[k]) / 2
    s2['nAllDots'] = s0['nAllDots'] + s1['nAllDots']
    s2['nTrimmedDots'] = s0['nTrimmedDots'] + s1['nTrimmedDots']
    s2['trimmedArea'] = s0['trimmedArea'] + s1['trimmedArea']
    return s2['s_median'], s2['trimmedArea'], s2['d_median'], dict(surface=surf, trimmed=trimmed,
                                                                      nn=extra)


# ----------------------------------------------------------------------------
# convenience entry points with the reference's argument conventions
# ----------------------------------------------------------------------------

def complex_inputs(binder_xyz, binder_radii, target_xyz, target_radii):
    """add_binder_and_target (_core.py:918-943): binder atoms then target atoms."""
    bx = np.asarray(binder_xyz, dtype=np.float64).reshape(-1, 3)
    tx = np.asarray(target_xyz, dtype=np.float64).reshape(-1, 3)
    xyz = np.concatenate([bx, tx])
    rad = np.concatenate([np.asarray(binder_radii, np.float64), np.asarray(target_radii, np.float64)])
    mol = np.concatenate([np.zeros(len(bx), np.int8), np.ones(len(tx), np.int8)])
    return xyz, rad, mol


def run_complex(binder_xyz, binder_radii, target_xyz, target_radii, settings=None, sc=True):
    """Surface + target CMS (+ binder CMS, SC) of one complex."""
    st = settings or Settings()
    xyz, rad, mol = complex_inputs(binder_xyz, binder_radii, target_xyz, target_radii)
    S = build_surface(xyz, rad, mol, st.density, st, all_atoms=False)
    out = dict(surface=S)
    out['cms'], out['cms_per_atom'] = contact_ms(S, True)
    out['cms_binder'], out['cms_binder_per_atom'] = contact_ms(S, False)
    if sc:
        out['sc'], out['sc_area'], out['sc_distance'], out['sc_details'] = shape_complementarity(S)
    return out


def run_max_cms(xyz, radii, settings=None):
    st = settings or Settings()
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    rad = np.asarray(radii, dtype=np.float64)
    S = build_surface(xyz, rad, np.zeros(len(rad), np.int8), st.density, st, all_atoms=True)
    tot, per = max_contact_ms(S)
    return tot, per, S
