/*
 * Seeded synthetic protein-like complexes for tests and benchmarks.
 *
 * A molecule of n heavy atoms is a self-avoiding random walk: 1.5 A steps in
 * random directions, confined to a sphere holding `vol_per_atom` cubic
 * Angstrom per atom, rejecting a step that lands closer than `min_nb` to any
 * atom other than the previous one.  When no direction works the clash
 * distance is relaxed by 5 % (never below `min_floor`) and the sphere grows by
 * 1 %, so the walk always completes; both relaxations are counted.
 *
 * A binder is rotated at random about its centroid and slid along a random
 * direction towards the target until the closest binder-target atom pair is
 * a gap drawn uniformly from [gap_lo, gap_hi].
 *
 * Everything is deterministic in the 64-bit seed (xoshiro256** seeded by
 * splitmix64).  Pure host C; the batch entry point runs molecules in parallel
 * with OpenMP.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void rng_seed(rng_t *r, uint64_t seed)
{
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&seed);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(rng_t *r)
{
    uint64_t *s = r->s;
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return result;
}

static double rng_uniform(rng_t *r) { return (rng_next(r) >> 11) * 0x1.0p-53; }

static void rng_unit(rng_t *r, double v[3])
{
    /* uniform direction: z uniform in [-1,1], azimuth uniform */
    double z = 2.0 * rng_uniform(r) - 1.0;
    double phi = 2.0 * M_PI * rng_uniform(r);
    double s = sqrt(fmax(0.0, 1.0 - z * z));
    v[0] = s * cos(phi); v[1] = s * sin(phi); v[2] = z;
}

/* ---- uniform grid over a cube, per-cell singly linked lists ------------- */
typedef struct {
    double lo, cell;
    int dim;
    int *head, *next;
} grid_t;

static int grid_init(grid_t *g, double half, double cell, int cap)
{
    g->cell = cell;
    g->lo = -half;
    g->dim = (int)ceil(2.0 * half / cell) + 1;
    if (g->dim < 1) g->dim = 1;
    size_t nc = (size_t)g->dim * g->dim * g->dim;
    g->head = (int *)malloc(nc * sizeof(int));
    g->next = (int *)malloc((size_t)(cap > 0 ? cap : 1) * sizeof(int));
    if (!g->head || !g->next) return -1;
    for (size_t i = 0; i < nc; ++i) g->head[i] = -1;
    return 0;
}

static void grid_free(grid_t *g) { free(g->head); free(g->next); }

static inline int gcoord(const grid_t *g, double x)
{
    int c = (int)floor((x - g->lo) / g->cell);
    return c < 0 ? 0 : (c >= g->dim ? g->dim - 1 : c);
}

static void grid_add(grid_t *g, const double *xyz, int i)
{
    int cx = gcoord(g, xyz[3 * i]), cy = gcoord(g, xyz[3 * i + 1]), cz = gcoord(g, xyz[3 * i + 2]);
    size_t c = ((size_t)cx * g->dim + cy) * g->dim + cz;
    g->next[i] = g->head[c];
    g->head[c] = i;
}

/* smallest squared distance from p to a stored atom other than `skip`, scanning
   cells within `reach` cells; returns +inf when nothing is in range */
static double grid_min_d2(const grid_t *g, const double *xyz, const double p[3], int skip, int reach)
{
    int cx = gcoord(g, p[0]), cy = gcoord(g, p[1]), cz = gcoord(g, p[2]);
    double best = INFINITY;
    for (int a = cx - reach; a <= cx + reach; ++a) {
        if (a < 0 || a >= g->dim) continue;
        for (int b = cy - reach; b <= cy + reach; ++b) {
            if (b < 0 || b >= g->dim) continue;
            for (int c = cz - reach; c <= cz + reach; ++c) {
                if (c < 0 || c >= g->dim) continue;
                for (int j = g->head[((size_t)a * g->dim + b) * g->dim + c]; j >= 0; j = g->next[j]) {
                    if (j == skip) continue;
                    double dx = p[0] - xyz[3 * j], dy = p[1] - xyz[3 * j + 1], dz = p[2] - xyz[3 * j + 2];
                    double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 < best) best = d2;
                }
            }
        }
    }
    return best;
}

/*
 * Random walk of n atoms.  Returns 0 on success, -1 on allocation failure.
 * stats (may be NULL): [0] clash relaxations, [1] sphere growths, [2] chain breaks.
 */
int cms_synth_walk(int n, uint64_t seed, double step, double min_nb, double min_floor,
                   double vol_per_atom, double *xyz, int64_t *stats)
{
    if (n <= 0) return 0;
    rng_t r;
    rng_seed(&r, seed);
    double R = cbrt(3.0 * vol_per_atom * n / (4.0 * M_PI));
    double half = 2.0 * R + 4.0 * step + 8.0;
    grid_t g;
    if (grid_init(&g, half, min_nb, n) != 0) { grid_free(&g); return -1; }
    int64_t relax = 0, grow = 0;
    {
        double v[3];
        rng_unit(&r, v);
        double f = 0.3 * R * rng_uniform(&r);
        xyz[0] = v[0] * f; xyz[1] = v[1] * f; xyz[2] = v[2] * f;
        grid_add(&g, xyz, 0);
    }
    const double Rmax = half - 2.0 * step - 2.0;
    int64_t breaks = 0;
    for (int i = 1; i < n; ++i) {
        double lim = min_nb;
        int placed = 0;
        for (;;) {
            for (int t = 0; t < 96 && !placed; ++t) {
                double v[3], p[3];
                rng_unit(&r, v);
                /* step length jittered by +-1 % so that no two bonded distances tie exactly */
                const double sl = step * (0.99 + 0.02 * rng_uniform(&r));
                p[0] = xyz[3 * (i - 1)] + sl * v[0];
                p[1] = xyz[3 * (i - 1) + 1] + sl * v[1];
                p[2] = xyz[3 * (i - 1) + 2] + sl * v[2];
                if (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > R * R) continue;
                if (fabs(p[0]) >= half - 1.0 || fabs(p[1]) >= half - 1.0 || fabs(p[2]) >= half - 1.0) continue;
                int reach = (int)ceil(lim / g.cell);
                if (grid_min_d2(&g, xyz, p, i - 1, reach) < lim * lim) continue;
                xyz[3 * i] = p[0]; xyz[3 * i + 1] = p[1]; xyz[3 * i + 2] = p[2];
                placed = 1;
            }
            if (placed) break;
            if (lim * 0.95 >= min_floor) { lim *= 0.95; ++relax; }
            else if (R < Rmax) { R = fmin(R * 1.01, Rmax); ++grow; }
            else break;
        }
        if (!placed) {
            /* dead end: break the chain and restart at a free point of the sphere */
            ++breaks;
            int reach = (int)ceil(min_floor / g.cell);
            for (int t = 0; t < 20000 && !placed; ++t) {
                double v[3], p[3];
                rng_unit(&r, v);
                double f = R * cbrt(rng_uniform(&r));
                p[0] = v[0] * f; p[1] = v[1] * f; p[2] = v[2] * f;
                if (grid_min_d2(&g, xyz, p, -1, reach) < min_floor * min_floor) continue;
                xyz[3 * i] = p[0]; xyz[3 * i + 1] = p[1]; xyz[3 * i + 2] = p[2];
                placed = 1;
            }
            if (!placed) {
                /* no free point found: a distinct point on a line outside the sphere */
                xyz[3 * i] = R + 3.0 + 2.5 * (double)breaks; xyz[3 * i + 1] = 0.0; xyz[3 * i + 2] = 0.0;
            }
        }
        grid_add(&g, xyz, i);
    }
    grid_free(&g);
    if (stats) { stats[0] = relax; stats[1] = grow; stats[2] = breaks; }
    return 0;
}

static void rand_rotation(rng_t *r, double m[9])
{
    /* uniform random unit quaternion (Shoemake) */
    double u1 = rng_uniform(r), u2 = rng_uniform(r), u3 = rng_uniform(r);
    double a = sqrt(1.0 - u1), b = sqrt(u1);
    double qw = a * sin(2 * M_PI * u2), qx = a * cos(2 * M_PI * u2);
    double qy = b * sin(2 * M_PI * u3), qz = b * cos(2 * M_PI * u3);
    m[0] = 1 - 2 * (qy * qy + qz * qz); m[1] = 2 * (qx * qy - qz * qw); m[2] = 2 * (qx * qz + qy * qw);
    m[3] = 2 * (qx * qy + qz * qw); m[4] = 1 - 2 * (qx * qx + qz * qz); m[5] = 2 * (qy * qz - qx * qw);
    m[6] = 2 * (qx * qz - qy * qw); m[7] = 2 * (qy * qz + qx * qw); m[8] = 1 - 2 * (qx * qx + qy * qy);
}

/* min binder-target distance, capped at `cap`, with the target in grid g */
static double contact_min(const grid_t *g, const double *txyz, const double *b, int nb,
                          const double off[3], double cap)
{
    double best = cap * cap;
    for (int i = 0; i < nb; ++i) {
        double p[3] = { b[3 * i] + off[0], b[3 * i + 1] + off[1], b[3 * i + 2] + off[2] };
        double d2 = grid_min_d2(g, txyz, p, -1, 1);
        if (d2 < best) best = d2;
    }
    return sqrt(best);
}

/*
 * Place a binder against a target.  bxyz/txyz are (n,3) row-major; the placed
 * binder is written to bout.  gap_out (may be NULL) receives the achieved
 * closest distance.  Returns 0, or -1 on allocation failure.
 */
int cms_synth_place(const double *bxyz, int nb, const double *txyz, int nt, uint64_t seed,
                    double gap_lo, double gap_hi, double *bout, double *gap_out)
{
    rng_t r;
    rng_seed(&r, seed);
    double cb[3] = {0, 0, 0}, ct[3] = {0, 0, 0};
    for (int i = 0; i < nb; ++i) for (int k = 0; k < 3; ++k) cb[k] += bxyz[3 * i + k] / nb;
    for (int i = 0; i < nt; ++i) for (int k = 0; k < 3; ++k) ct[k] += txyz[3 * i + k] / nt;
    double m[9];
    rand_rotation(&r, m);
    double *rb = (double *)malloc((size_t)(nb > 0 ? nb : 1) * 3 * sizeof(double));
    if (!rb) return -1;
    double Rb = 0, Rt = 0;
    for (int i = 0; i < nb; ++i) {
        double v[3] = { bxyz[3 * i] - cb[0], bxyz[3 * i + 1] - cb[1], bxyz[3 * i + 2] - cb[2] };
        for (int k = 0; k < 3; ++k) rb[3 * i + k] = m[3 * k] * v[0] + m[3 * k + 1] * v[1] + m[3 * k + 2] * v[2];
        double d = sqrt(rb[3 * i] * rb[3 * i] + rb[3 * i + 1] * rb[3 * i + 1] + rb[3 * i + 2] * rb[3 * i + 2]);
        if (d > Rb) Rb = d;
    }
    /* target relative to its centroid, in a grid with 5 A cells */
    double *tt = (double *)malloc((size_t)(nt > 0 ? nt : 1) * 3 * sizeof(double));
    if (!tt) { free(rb); return -1; }
    for (int i = 0; i < nt; ++i) {
        for (int k = 0; k < 3; ++k) tt[3 * i + k] = txyz[3 * i + k] - ct[k];
        double d = sqrt(tt[3 * i] * tt[3 * i] + tt[3 * i + 1] * tt[3 * i + 1] + tt[3 * i + 2] * tt[3 * i + 2]);
        if (d > Rt) Rt = d;
    }
    const double cap = 5.0;
    grid_t g;
    if (grid_init(&g, Rt + 2 * cap, cap, nt) != 0) { grid_free(&g); free(rb); free(tt); return -1; }
    for (int i = 0; i < nt; ++i) grid_add(&g, tt, i);
    double u[3];
    rng_unit(&r, u);
    double gap = gap_lo + (gap_hi - gap_lo) * rng_uniform(&r);
    double hi = Rt + Rb + cap + 1.0, lo = hi;
    double off[3];
    /* walk in until the closest pair is nearer than the gap */
    for (;;) {
        lo = hi - 0.5;
        if (lo < 0) { lo = 0; break; }
        off[0] = u[0] * lo; off[1] = u[1] * lo; off[2] = u[2] * lo;
        if (contact_min(&g, tt, rb, nb, off, cap) < gap) break;
        hi = lo;
    }
    for (int it = 0; it < 50; ++it) {
        double mid = 0.5 * (lo + hi);
        off[0] = u[0] * mid; off[1] = u[1] * mid; off[2] = u[2] * mid;
        if (contact_min(&g, tt, rb, nb, off, cap) < gap) lo = mid; else hi = mid;
    }
    off[0] = u[0] * hi; off[1] = u[1] * hi; off[2] = u[2] * hi;
    if (gap_out) *gap_out = contact_min(&g, tt, rb, nb, off, cap);
    for (int i = 0; i < nb; ++i)
        for (int k = 0; k < 3; ++k) bout[3 * i + k] = rb[3 * i + k] + off[k] + ct[k];
    grid_free(&g);
    free(rb);
    free(tt);
    return 0;
}

/*
 * One complex cut from a single globule: a walk of nt + nb atoms, split by a
 * plane with a random normal u into the nb atoms furthest along u (binder)
 * and the rest (target); the binder is then slid out along u until its
 * closest target atom is `gap` away.  The two faces are complementary, so the
 * interface spans the whole cut.  Output order: binder atoms then target
 * atoms, each in walk order; perm[k] is the walk index of output atom k.
 */
static int cmp_key(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x < y) ? -1 : (x > y);
}

int cms_synth_cut(int nt, int nb, uint64_t seed, double step, double min_nb, double min_floor,
                  double vol_per_atom, double gap_lo, double gap_hi, double *out, int *perm, double *gap_out)
{
    const int n = nt + nb;
    if (n <= 0) return 0;
    uint64_t s = seed;
    uint64_t sw = splitmix64(&s), sp = splitmix64(&s);
    double *w = (double *)malloc((size_t)n * 3 * sizeof(double));
    double *key = (double *)malloc((size_t)n * 2 * sizeof(double));
    char *isb = (char *)calloc((size_t)n, 1);
    if (!w || !key || !isb) { free(w); free(key); free(isb); return -1; }
    if (cms_synth_walk(n, sw, step, min_nb, min_floor, vol_per_atom, w, NULL) != 0) {
        free(w); free(key); free(isb); return -1;
    }
    rng_t r;
    rng_seed(&r, sp);
    double u[3];
    rng_unit(&r, u);
    for (int i = 0; i < n; ++i) {
        key[2 * i] = w[3 * i] * u[0] + w[3 * i + 1] * u[1] + w[3 * i + 2] * u[2];
        key[2 * i + 1] = (double)i;
    }
    qsort(key, (size_t)n, 2 * sizeof(double), cmp_key);
    for (int k = n - nb; k < n; ++k) isb[(int)key[2 * k + 1]] = 1;
    int kb = 0, kt = nb;
    for (int i = 0; i < n; ++i) {
        int k = isb[i] ? kb++ : kt++;
        perm[k] = i;
        for (int a = 0; a < 3; ++a) out[3 * k + a] = w[3 * i + a];
    }
    double gap = gap_lo + (gap_hi - gap_lo) * rng_uniform(&r);
    double achieved = 0.0;
    if (nb > 0 && nt > 0) {
        /* target in a grid; slide the binder along u */
        double Rt = 0.0;
        for (int i = nb; i < n; ++i)
            Rt = fmax(Rt, sqrt(out[3 * i] * out[3 * i] + out[3 * i + 1] * out[3 * i + 1] + out[3 * i + 2] * out[3 * i + 2]));
        const double cap = 6.0;
        grid_t g;
        if (grid_init(&g, Rt + 2 * cap + 4.0, cap, nt) != 0) { grid_free(&g); free(w); free(key); free(isb); return -1; }
        for (int i = 0; i < nt; ++i) grid_add(&g, out + 3 * nb, i);
        double off[3], lo = 0.0, hi = 1.0;
        for (;;) {
            off[0] = u[0] * hi; off[1] = u[1] * hi; off[2] = u[2] * hi;
            if (contact_min(&g, out + 3 * nb, out, nb, off, cap) >= gap || hi > 64.0) break;
            lo = hi; hi *= 2.0;
        }
        for (int it = 0; it < 60; ++it) {
            double mid = 0.5 * (lo + hi);
            off[0] = u[0] * mid; off[1] = u[1] * mid; off[2] = u[2] * mid;
            if (contact_min(&g, out + 3 * nb, out, nb, off, cap) < gap) lo = mid; else hi = mid;
        }
        off[0] = u[0] * hi; off[1] = u[1] * hi; off[2] = u[2] * hi;
        achieved = contact_min(&g, out + 3 * nb, out, nb, off, cap);
        for (int i = 0; i < nb; ++i)
            for (int a = 0; a < 3; ++a) out[3 * i + a] += off[a];
        grid_free(&g);
    }
    if (gap_out) *gap_out = achieved;
    free(w); free(key); free(isb);
    return 0;
}

/*
 * Batch of complexes: molecule sizes n_target[c], n_binder[c]; the outputs are
 * concatenated per complex as binder atoms then target atoms, starting at
 * atom_off[c] (atom_off has B+1 entries); perm receives, per complex, the walk
 * index of each output atom.  seeds[c] seeds complex c.  Returns 0 or the
 * first nonzero status.
 */
int cms_synth_batch(int B, const int *n_target, const int *n_binder, const uint64_t *seeds,
                    const int64_t *atom_off, double step, double min_nb, double min_floor,
                    double vol_per_atom, double gap_lo, double gap_hi, double *xyz, int *perm, double *gaps)
{
    int status = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : status)
    for (int c = 0; c < B; ++c) {
        double gap = 0.0;
        int e = cms_synth_cut(n_target[c], n_binder[c], seeds[c], step, min_nb, min_floor, vol_per_atom,
                              gap_lo, gap_hi, xyz + 3 * atom_off[c], perm + atom_off[c], &gap);
        if (gaps) gaps[c] = gap;
        status |= (e != 0);
    }
    return status;
}
