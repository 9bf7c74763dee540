/*
 * sl_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * CPU restatement, in plain C, of slChannel's semi-Lagrangian trace and
 * tensor-product Lagrange gather (slchannel/semilag.py of gmcavallazzi/SLchannel
 * v1.0.1, the eager float64 path).  Every function cites the reference lines it
 * follows, and keeps the reference's order of floating-point operations, so its
 * output agrees with the reference's eager torch path to the last few ulps.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm may load this library, and only as the reference answer that results are
 * compared against or as the timed CPU baseline;
 * the product path (slchannel_b200) never calls it.
 *
 * Threads: POSIX threads over contiguous ranges of arrival points (each point
 * is independent; the clamp count is an integer sum, so results do not depend
 * on the thread count).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_MAX_ORDER 6

/* One component's node grid (semilag.py:87-99 _GridSpec).  dinv[o] is the
 * inverse-denominator table for stencil order o, shape (NZ - o + 1, o),
 * row-major (semilag.py:102-114). */
typedef struct {
    int64_t NX, NY, NZ;
    double shift_x, shift_y;
    int32_t centers; /* 1: z nodes are cell centres incl. ghosts; 0: faces */
    int32_t pad_;
    const double *znodes;
    const double *dinv[ORC_MAX_ORDER + 1];
} orc_spec;

typedef struct {
    int64_t nx, ny, nz;
    double dx, dy, Lz, gamma, tanh_g, z_lo, z_hi;
    int32_t symmetric;
    int32_t n_traj_iters;
    int32_t traj_order;
    int32_t order;
    double udenom[ORC_MAX_ORDER + 1][ORC_MAX_ORDER]; /* semilag.py:117-127 */
    const double *z_c; /* nz + 2 */
    const double *z_f; /* nz + 1 */
    orc_spec spec[3];
} orc_grid;

static int g_threads = 0;

void orc_set_threads(int n) { g_threads = n; }

int orc_max_threads(void)
{
    if (g_threads > 0) return g_threads;
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* Static-schedule parallel for: body(ctx, p0, p1) over [0, n), returns the
 * sum of the per-range integer results. */
typedef int64_t (*range_fn)(void *ctx, int64_t p0, int64_t p1);
typedef struct {
    range_fn fn;
    void *ctx;
    int64_t p0, p1, result;
} range_job;

static void *range_worker(void *arg)
{
    range_job *j = (range_job *)arg;
    j->result = j->fn(j->ctx, j->p0, j->p1);
    return NULL;
}

static int64_t parallel_for(int64_t n, range_fn fn, void *ctx)
{
    int nt = orc_max_threads();
    if (nt > 256) nt = 256;
    if (n < 4096 || nt <= 1) return fn(ctx, 0, n);
    range_job jobs[256];
    pthread_t th[256];
    int64_t chunk = (n + nt - 1) / nt;
    int started = 0;
    for (int t = 0; t < nt; ++t) {
        int64_t a = t * chunk, b = a + chunk < n ? a + chunk : n;
        if (a >= b) break;
        jobs[t] = (range_job){fn, ctx, a, b, 0};
        if (pthread_create(&th[t], NULL, range_worker, &jobs[t]) != 0) {
            jobs[t].result = fn(ctx, a, b);
            th[t] = 0;
        }
        started = t + 1;
    }
    int64_t total = 0;
    for (int t = 0; t < started; ++t) {
        if (th[t]) pthread_join(th[t], NULL);
        total += jobs[t].result;
    }
    return total;
}

/* semilag.py:400-411 _face_coord */
static double face_coord(const orc_grid *g, double z)
{
    const double lo = -1.0 + 1e-15, hi = 1.0 - 1e-15;
    if (g->symmetric) {
        double arg = (2.0 * z / g->Lz - 1.0) * g->tanh_g;
        if (arg < lo) arg = lo;
        if (arg > hi) arg = hi;
        double xi = atanh(arg) / g->gamma;
        return (xi + 1.0) * (0.5 * (double)g->nz);
    } else {
        double arg = (1.0 - z / g->Lz) * g->tanh_g;
        if (arg < lo) arg = lo;
        if (arg > hi) arg = hi;
        double xi = 1.0 - atanh(arg) / g->gamma;
        return xi * (double)g->nz;
    }
}

/* semilag.py:413-420 _locate_z */
static int64_t locate_z(const orc_grid *g, const orc_spec *s, double z)
{
    double kf = face_coord(g, z);
    int64_t c = (int64_t)floor(kf);
    if (c < 0) c = 0;
    if (c > g->nz - 1) c = g->nz - 1;
    if (!s->centers) return c;
    return c + (z >= s->znodes[c + 1] ? 1 : 0);
}

static int64_t pmod(int64_t a, int64_t n)
{
    int64_t r = a % n;
    return r < 0 ? r + n : r;
}

/* semilag.py:426-439 _uniform_weights: Lagrange weights on integer offsets
 * off_m = m - (order/2 - 1), numerator product in ascending l. */
static void uniform_weights(const orc_grid *g, double t, int order, double *w)
{
    const int h = order / 2 - 1;
    double d[ORC_MAX_ORDER];
    for (int l = 0; l < order; ++l) d[l] = t - (double)(l - h);
    for (int m = 0; m < order; ++m) {
        double num = 0.0;
        int first = 1;
        for (int l = 0; l < order; ++l) {
            if (l == m) continue;
            if (first) { num = d[l]; first = 0; }
            else num = num * d[l];
        }
        w[m] = num * g->udenom[order][m];
    }
}

/* semilag.py:441-454 _z_weights */
static void z_weights(const orc_spec *s, double z, int64_t k0, int order, double *w)
{
    double d[ORC_MAX_ORDER];
    for (int l = 0; l < order; ++l) d[l] = z - s->znodes[k0 + l];
    const double *dinv = s->dinv[order] + k0 * order;
    for (int m = 0; m < order; ++m) {
        double num = 0.0;
        int first = 1;
        for (int l = 0; l < order; ++l) {
            if (l == m) continue;
            if (first) { num = d[l]; first = 0; }
            else num = num * d[l];
        }
        w[m] = num * dinv[m];
    }
}

typedef struct {
    int64_t ixl[ORC_MAX_ORDER], iyl[ORC_MAX_ORDER], k0;
    double wx[ORC_MAX_ORDER], wy[ORC_MAX_ORDER], wz[ORC_MAX_ORDER];
} stencil_t;

/* semilag.py:471-500 _build_iw_impl for one point (z already clamped). */
static void build_stencil(const orc_grid *g, const orc_spec *s, int order, double x, double y,
                          double z, stencil_t *st)
{
    const int h = order / 2 - 1;
    double sx = x / g->dx + s->shift_x;
    double ix0 = floor(sx);
    double tx = sx - ix0;
    for (int m = 0; m < order; ++m)
        st->ixl[m] = pmod((int64_t)ix0 + (m - h), s->NX) * (s->NY * s->NZ);
    uniform_weights(g, tx, order, st->wx);

    double sy = y / g->dy + s->shift_y;
    double iy0 = floor(sy);
    double ty = sy - iy0;
    for (int m = 0; m < order; ++m) st->iyl[m] = pmod((int64_t)iy0 + (m - h), s->NY) * s->NZ;
    uniform_weights(g, ty, order, st->wy);

    int64_t m0 = locate_z(g, s, z);
    int64_t k0 = m0 - h;
    if (k0 < 0) k0 = 0;
    if (k0 > s->NZ - order) k0 = s->NZ - order;
    st->k0 = k0;
    z_weights(s, z, k0, order, st->wz);
}

/* semilag.py:44-59 _gather_interp: sequential accumulation in (i, j, k). */
static double gather(const double *F, const stencil_t *st, int order)
{
    double out = 0.0;
    int first = 1;
    for (int i = 0; i < order; ++i) {
        for (int j = 0; j < order; ++j) {
            int64_t base = st->ixl[i] + st->iyl[j] + st->k0;
            double wij = st->wx[i] * st->wy[j];
            for (int k = 0; k < order; ++k) {
                double term = (wij * st->wz[k]) * F[base + k];
                if (first) { out = term; first = 0; }
                else out = out + term;
            }
        }
    }
    return out;
}

static double clampd(double v, double lo, double hi)
{
    /* torch.clamp(min, max) */
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

/* semilag.py:512-528 _sample: trajectory velocity at one point. */
static double sample(const orc_grid *g, int comp, const double *mbuf, double x, double y, double z)
{
    stencil_t st;
    build_stencil(g, &g->spec[comp], g->traj_order, x, y, clampd(z, g->z_lo, g->z_hi), &st);
    return gather(mbuf, &st, g->traj_order);
}

/* semilag.py:292-307 arrival coordinates of flat interior point p. */
static void arrival(const orc_grid *g, int comp, int64_t p, double *xa, double *ya, double *za)
{
    int64_t nzi = comp == 2 ? g->nz - 1 : g->nz;
    int64_t k = p % nzi;
    int64_t j = (p / nzi) % g->ny;
    int64_t i = p / (nzi * g->ny);
    double ar = (double)(i + 1), aj = (double)(j + 1);
    if (comp == 0) {
        *xa = ar * g->dx;
        *ya = (aj - 0.5) * g->dy;
        *za = g->z_c[k + 1];
    } else if (comp == 1) {
        *xa = (ar - 0.5) * g->dx;
        *ya = aj * g->dy;
        *za = g->z_c[k + 1];
    } else {
        *xa = (ar - 0.5) * g->dx;
        *ya = (aj - 0.5) * g->dy;
        *za = g->z_f[k + 1];
    }
}

/* semilag.py:534-552 departure_coords for one arrival point. */
static void departure(const orc_grid *g, const double *const mid[3], double dt, double xa, double ya,
                      double za, double *xd, double *yd, double *zd)
{
    double half_dt = 0.5 * dt;
    double xm = xa, ym = ya, zm = za;
    for (int it = 0; it < g->n_traj_iters; ++it) {
        double us = sample(g, 0, mid[0], xm, ym, zm);
        double vs = sample(g, 1, mid[1], xm, ym, zm);
        double ws = sample(g, 2, mid[2], xm, ym, zm);
        xm = xa - half_dt * us;
        ym = ya - half_dt * vs;
        zm = clampd(za - half_dt * ws, g->z_lo, g->z_hi);
    }
    *xd = 2.0 * xm - xa;
    *yd = 2.0 * ym - ya;
    *zd = 2.0 * zm - za;
}

int64_t orc_n_arrival(const orc_grid *g, int comp)
{
    return g->nx * g->ny * (comp == 2 ? g->nz - 1 : g->nz);
}

/* semilag.py:400-411, vectorised over n points. */
typedef struct {
    const orc_grid *g;
    const double *z;
    double *kf;
} fc_ctx;

static int64_t fc_range(void *c, int64_t p0, int64_t p1)
{
    fc_ctx *x = (fc_ctx *)c;
    for (int64_t p = p0; p < p1; ++p) x->kf[p] = face_coord(x->g, x->z[p]);
    return 0;
}

void orc_face_coord(const orc_grid *g, const double *z, int64_t n, double *kf)
{
    fc_ctx c = {g, z, kf};
    parallel_for(n, fc_range, &c);
}

/* semilag.py:460-510 _build_iw + _apply_iw at n arbitrary points.  With
 * count_clamp, z is clamped to [z_lo, z_hi] and the clamps are counted
 * (semilag.py:472-474); returns the count. */
typedef struct {
    const orc_grid *g;
    int comp, order, count_clamp;
    const double *buf, *x, *y, *z;
    double *out;
} interp_ctx;

static int64_t interp_range(void *c, int64_t p0, int64_t p1)
{
    interp_ctx *a = (interp_ctx *)c;
    int64_t ncl = 0;
    for (int64_t p = p0; p < p1; ++p) {
        double zz = a->z[p];
        if (a->count_clamp) {
            if (zz < a->g->z_lo || zz > a->g->z_hi) ncl += 1;
            zz = clampd(zz, a->g->z_lo, a->g->z_hi);
        }
        stencil_t st;
        build_stencil(a->g, &a->g->spec[a->comp], a->order, a->x[p], a->y[p], zz, &st);
        a->out[p] = gather(a->buf, &st, a->order);
    }
    return ncl;
}

int64_t orc_interp(const orc_grid *g, int comp, int order, const double *buf, const double *x,
                   const double *y, const double *z, int64_t n, int count_clamp, double *out)
{
    interp_ctx c = {g, comp, order, count_clamp, buf, x, y, z, out};
    return parallel_for(n, interp_range, &c);
}

/* semilag.py:534-552 over every arrival point of `comp`. */
typedef struct {
    const orc_grid *g;
    int comp;
    const double *mid[3];
    const double *fbuf;
    double dt;
    int64_t p0;
    double *xd, *yd, *zd, *out;
} adv_ctx;

static int64_t dep_range(void *c, int64_t p0, int64_t p1)
{
    adv_ctx *a = (adv_ctx *)c;
    for (int64_t p = p0; p < p1; ++p) {
        double xa, ya, za;
        arrival(a->g, a->comp, p, &xa, &ya, &za);
        departure(a->g, a->mid, a->dt, xa, ya, za, &a->xd[p], &a->yd[p], &a->zd[p]);
    }
    return 0;
}

void orc_departure(const orc_grid *g, int comp, const double *mu, const double *mv, const double *mw,
                   double dt, double *xd, double *yd, double *zd)
{
    adv_ctx c = {g, comp, {mu, mv, mw}, NULL, dt, 0, xd, yd, zd, NULL};
    parallel_for(orc_n_arrival(g, comp), dep_range, &c);
}

/* semilag.py:560-571 _advect_comp_impl (eager equivalent): departure point,
 * clamped and counted stencil at `order`, gather of the node buffer `fbuf`.
 * Arrival points p in [p0, p1) only (a bounded sample for CPU timing uses a
 * sub-range; the full call passes 0, n).  Returns the clamp count. */
static int64_t adv_range(void *c, int64_t q0, int64_t q1)
{
    adv_ctx *a = (adv_ctx *)c;
    const orc_grid *g = a->g;
    int64_t ncl = 0;
    for (int64_t q = q0; q < q1; ++q) {
        int64_t p = a->p0 + q;
        double xa, ya, za, xd, yd, zd;
        arrival(g, a->comp, p, &xa, &ya, &za);
        departure(g, a->mid, a->dt, xa, ya, za, &xd, &yd, &zd);
        if (zd < g->z_lo || zd > g->z_hi) ncl += 1;
        zd = clampd(zd, g->z_lo, g->z_hi);
        stencil_t st;
        build_stencil(g, &g->spec[a->comp], g->order, xd, yd, zd, &st);
        a->out[q] = gather(a->fbuf, &st, g->order);
    }
    return ncl;
}

int64_t orc_advect_comp_range(const orc_grid *g, int comp, const double *fbuf, const double *mu,
                              const double *mv, const double *mw, double dt, int64_t p0,
                              int64_t p1, double *out)
{
    adv_ctx c = {g, comp, {mu, mv, mw}, fbuf, dt, p0, NULL, NULL, NULL, out};
    return parallel_for(p1 - p0, adv_range, &c);
}

int64_t orc_advect_comp(const orc_grid *g, int comp, const double *fbuf, const double *mu,
                        const double *mv, const double *mw, double dt, double *out)
{
    return orc_advect_comp_range(g, comp, fbuf, mu, mv, mw, dt, 0, orc_n_arrival(g, comp), out);
}

/* ---------------------------------------------------------------------------
 * tridiag.py:36-61 pcr_solve for a batch of right-hand sides sharing the 1-D
 * diagonals a, b, c (length n); d is (batch, n), solved in place.  The
 * diagonals evolve the same way for every system, so their levels are
 * computed once; each system then takes the same per-level update
 *   d <- (d + alpha * d[i-s]) + gamma * d[i+s]    (absent neighbours 0)
 * and x = d / b, in the reference's operation order (no contraction).
 * ------------------------------------------------------------------------- */
typedef struct {
    const double *alpha, *gamma, *bfin;  /* levels x n, levels x n, n */
    double *d;
    int n, levels;
} pcr_ctx;

static int64_t pcr_range(void *c, int64_t r0, int64_t r1)
{
    pcr_ctx *p = (pcr_ctx *)c;
    const int n = p->n;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
    if (!tmp) return -1;
    for (int64_t r = r0; r < r1; ++r) {
        double *d = p->d + r * (int64_t)n;
        int s = 1;
        for (int l = 0; l < p->levels; ++l, s *= 2) {
            const double *al = p->alpha + (size_t)l * n, *ga = p->gamma + (size_t)l * n;
            for (int i = 0; i < n; ++i) {
                const double dd = i - s >= 0 ? d[i - s] : 0.0;
                const double du = i + s < n ? d[i + s] : 0.0;
                const double t1 = al[i] * dd;
                const double t2 = d[i] + t1;
                const double t3 = ga[i] * du;
                tmp[i] = t2 + t3;
            }
            memcpy(d, tmp, sizeof(double) * (size_t)n);
        }
        for (int i = 0; i < n; ++i) d[i] = d[i] / p->bfin[i];
    }
    free(tmp);
    return 0;
}

int orc_pcr_batch(const double *a0, const double *b0, const double *c0, double *d, int64_t batch,
                  int n)
{
    if (n < 1 || batch < 0) return 1;
    int levels = 0;
    for (int s = 1; s < n; s *= 2) ++levels;
    double *a = (double *)malloc(sizeof(double) * (size_t)n * 8);
    double *alpha = (double *)malloc(sizeof(double) * (size_t)n * (levels + 1));
    double *gamma = (double *)malloc(sizeof(double) * (size_t)n * (levels + 1));
    if (!a || !alpha || !gamma) {
        free(a); free(alpha); free(gamma);
        return 2;
    }
    double *b = a + n, *c = b + n, *na = c + n, *nb = na + n, *nc = nb + n;
    memcpy(a, a0, sizeof(double) * (size_t)n);
    memcpy(b, b0, sizeof(double) * (size_t)n);
    memcpy(c, c0, sizeof(double) * (size_t)n);
    int s = 1;
    for (int l = 0; l < levels; ++l, s *= 2) {
        double *al = alpha + (size_t)l * n, *ga = gamma + (size_t)l * n;
        for (int i = 0; i < n; ++i) {
            const int dn = i - s, up = i + s;
            const double a_dn = dn >= 0 ? a[dn] : 0.0, b_dn = dn >= 0 ? b[dn] : 1.0;
            const double c_dn = dn >= 0 ? c[dn] : 0.0;
            const double a_up = up < n ? a[up] : 0.0, b_up = up < n ? b[up] : 1.0;
            const double c_up = up < n ? c[up] : 0.0;
            const double alp = -a[i] / b_dn;
            const double gam = -c[i] / b_up;
            const double t1 = alp * c_dn;
            const double t2 = b[i] + t1;
            const double t3 = gam * a_up;
            nb[i] = t2 + t3;
            na[i] = alp * a_dn;
            nc[i] = gam * c_up;
            al[i] = alp;
            ga[i] = gam;
        }
        memcpy(a, na, sizeof(double) * (size_t)n);
        memcpy(b, nb, sizeof(double) * (size_t)n);
        memcpy(c, nc, sizeof(double) * (size_t)n);
    }
    pcr_ctx ctx = {alpha, gamma, b, d, n, levels};
    int64_t rc = parallel_for(batch, pcr_range, &ctx);
    free(a); free(alpha); free(gamma);
    return rc < 0 ? 3 : 0;
}
