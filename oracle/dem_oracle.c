/*
 * CPU oracle for the sphere DEM step -- TEST INFRASTRUCTURE ONLY (see
 * sph_oracle.h).  Every function cites the reference kernel it restates.
 * Compile with -ffp-contract=off and without -ffast-math.
 */
#include "sph_oracle.h"
#include "oracle_internal.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* vector helpers: same operation order as src/vector_arithmetic.h      */
/* ------------------------------------------------------------------ */
static inline v3 mk3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
/* Float * Float3 (vector_arithmetic.h: b * a.x) */
static inline v3 smul3(double b, v3 a) { return mk3(b * a.x, b * a.y, b * a.z); }
/* Float3 * Float (a.x * b) */
static inline v3 muls3(v3 a, double b) { return mk3(a.x * b, a.y * b, a.z * b); }
static inline v3 divs3(v3 a, double b) { return mk3(a.x / b, a.y / b, a.z / b); }
static inline v3 adds3(v3 a, double b) { return mk3(a.x + b, a.y + b, a.z + b); }
static inline double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 xyz(d4 a) { return mk3(a.x, a.y, a.z); }

/* length(): src/vector_arithmetic.h:317-324.  Faithful mode rounds the FP64
 * dot product to FP32 and takes the IEEE FP32 square root. */
double orc_len(const orc_state *s, v3 v)
{
    double d = dot3(v, v);
    if (s->precision == 0)
        return (double)sqrtf((float)d);
    return sqrt(d);
}

/* sqrtf of a Float argument used directly in the kernels
 * (contactmodels.cuh:196,341, cohesion.cuh:260-269). */
double orc_sqrtf(const orc_state *s, double v)
{
    if (s->precision == 0)
        return (double)sqrtf((float)v);
    return sqrt(v);
}

void orc_set_error(orc_state *s, int code, const char *msg)
{
#pragma omp critical(orc_error)
    {
        if (s->err == 0) {
            s->err = code;
            snprintf(s->errmsg, sizeof(s->errmsg), "%s", msg);
        }
    }
}

/* ------------------------------------------------------------------ */
/* a1: cell hashing, src/sorting.cuh:7-51                               */
/* ------------------------------------------------------------------ */
static int cell_coord(const orc_state *s, double x, int d, int64_t *out)
{
    double f = floor((x - s->origo[d]) / (s->L[d] / s->num[d]));
    if (!(f >= 0.0) || f >= (double)s->num[d])
        return -1;
    *out = (int64_t)f;
    return 0;
}

static int stage_hash(orc_state *s)
{
    for (unsigned i = 0; i < s->np; ++i) {
        int64_t ix, iy, iz;
        d4 x = s->x[i];
        if (cell_coord(s, x.x, 0, &ix) || cell_coord(s, x.y, 1, &iy) ||
            cell_coord(s, x.z, 2, &iz)) {
            char m[160];
            snprintf(m, sizeof m, "particle %u at (%g, %g, %g) is outside the "
                     "grid or not finite", i, x.x, x.y, x.z);
            orc_set_error(s, ORC_ERR_OUTSIDE, m);
            return ORC_ERR_OUTSIDE;
        }
        s->cellid[i] = (unsigned)((iz * s->num[1]) * s->num[0] + iy * s->num[0] + ix);
        s->index[i] = i;
    }
    return 0;
}

/* a2: thrust::sort_by_key (device.cu:1082-1085) is a stable key sort; a
 * counting sort over cells that visits particles in index order gives the
 * same permutation. */
static void stage_sort(orc_state *s)
{
    unsigned nc = s->ncells;
    unsigned *count = s->sort_count;
    memset(count, 0, sizeof(unsigned) * (nc + 1));
    for (unsigned i = 0; i < s->np; ++i) count[s->cellid[i] + 1]++;
    for (unsigned c = 0; c < nc; ++c) count[c + 1] += count[c];
    for (unsigned i = 0; i < s->np; ++i) {
        unsigned c = s->cellid[i];
        unsigned pos = count[c]++;
        s->sort_key[pos] = c;
        s->sort_val[pos] = i;
    }
    memcpy(s->cellid, s->sort_key, sizeof(unsigned) * s->np);
    memcpy(s->index, s->sort_val, sizeof(unsigned) * s->np);
}

/* a3: cellStart sentinel memset (device.cu:1096-1097) + reorderArrays
 * (sorting.cuh:56-132). cellEnd is never reset by the reference. */
static void stage_reorder(orc_state *s)
{
    for (unsigned c = 0; c < s->ncells; ++c) s->cellstart[c] = 0xffffffffu;
    for (unsigned i = 0; i < s->np; ++i) {
        unsigned cell = s->cellid[i];
        if (i == 0 || cell != s->cellid[i - 1]) {
            s->cellstart[cell] = i;
            if (i > 0) s->cellend[s->cellid[i - 1]] = i;
        }
        if (i == s->np - 1) s->cellend[cell] = i + 1;
        unsigned o = s->index[i];
        s->x_sorted[i] = s->x[o];
        s->vel_sorted[i] = s->vel[o];
        s->angvel_sorted[i] = s->angvel[o];
    }
}

int orc_stage_hash_sort_reorder(orc_state *s)
{
    int rc = stage_hash(s);
    if (rc) return rc;
    stage_sort(s);
    stage_reorder(s);
    return 0;
}

/* ------------------------------------------------------------------ */
/* a4: findDistMod, src/contactsearch.cuh:12-83                         */
/* ------------------------------------------------------------------ */
static int find_distmod(const orc_state *s, int *cx, int *cy, int *cz, v3 *dm)
{
    int nx = (int)s->num[0], ny = (int)s->num[1], nz = (int)s->num[2];
    if (s->periodic == 1) {
        if (*cx < 0) { *cx += nx; *dm = add3(*dm, mk3(s->L[0], 0.0, 0.0)); }
        if (*cx >= nx) { *cx -= nx; *dm = sub3(*dm, mk3(s->L[0], 0.0, 0.0)); }
        if (*cy < 0) { *cy += ny; *dm = add3(*dm, mk3(0.0, s->L[1], 0.0)); }
        if (*cy >= ny) { *cy -= ny; *dm = sub3(*dm, mk3(0.0, s->L[1], 0.0)); }
    }
    if (s->periodic == 2) {
        if (*cx < 0) { *cx += nx; *dm = add3(*dm, mk3(s->L[0], 0.0, 0.0)); }
        if (*cx >= nx) { *cx -= nx; *dm = sub3(*dm, mk3(s->L[0], 0.0, 0.0)); }
        if (*cy < 0 || *cy >= ny) return -1;
    }
    if (s->periodic > 2 || s->periodic < 1) {
        if (*cx < 0 || *cx >= nx) return -1;
        if (*cy < 0 || *cy >= ny) return -1;
    }
    if (*cz < 0 || *cz >= nz) return -1;
    return 0;
}

static void grid_pos(const orc_state *s, d4 x, int *gx, int *gy, int *gz)
{
    *gx = (int)floor((x.x - s->origo[0]) / (s->L[0] / s->num[0]));
    *gy = (int)floor((x.y - s->origo[1]) / (s->L[1] / s->num[1]));
    *gz = (int)floor((x.z - s->origo[2]) / (s->L[2] / s->num[2]));
}

/* ------------------------------------------------------------------ */
/* a5: topology + findContactsInCell, src/contactsearch.cuh:194-371     */
/* ------------------------------------------------------------------ */
static void topology_particle(orc_state *s, unsigned a)
{
    d4 xa = s->x_sorted[a];
    double ra = xa.w;
    unsigned a_orig = s->index[a];
    unsigned NCs = s->nc;
    unsigned *row = s->contacts + (size_t)a_orig * NCs;
    int nc = 0;
    int gx, gy, gz;
    grid_pos(s, xa, &gx, &gy, &gz);
    for (int dz = -1; dz < 2; ++dz)
        for (int dy = -1; dy < 2; ++dy)
            for (int dx = -1; dx < 2; ++dx) {
                int cx = gx + dx, cy = gy + dy, cz = gz + dz;
                v3 dm = mk3(0.0, 0.0, 0.0);
                if (find_distmod(s, &cx, &cy, &cz, &dm) == -1) continue;
                unsigned cell = (unsigned)cx + (unsigned)cy * s->num[0] +
                                (s->num[0] * s->num[1]) * (unsigned)cz;
                unsigned start = s->cellstart[cell];
                if (start == 0xffffffffu) continue;
                unsigned end = s->cellend[cell];
                for (unsigned b = start; b < end; ++b) {
                    if (b == a) continue;
                    d4 xb = s->x_sorted[b];
                    double rb = xb.w;
                    unsigned b_orig = s->index[b];
                    v3 xab = mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
                    xab = add3(xab, dm);
                    double len = orc_len(s, xab);
                    double delta = len - (ra + rb);
                    if (delta < 0.0) {
                        int cpos = nc;
                        for (unsigned i = 0; i < NCs; ++i) {
                            unsigned c = row[i];
                            if (c == s->np) cpos = (int)i;
                            else if (c == b_orig) { cpos = (int)i; break; }
                        }
                        if (cpos >= (int)NCs) {
                            /* The reference writes outside this particle's
                             * slot row here; report it instead. */
                            orc_set_error(s, ORC_ERR_CAPACITY,
                                          "contact slot capacity exceeded");
                            return;
                        }
                        row[cpos] = b_orig;
                        d4 dmv = {dm.x, dm.y, dm.z, rb};
                        s->distmod[(size_t)a_orig * NCs + cpos] = dmv;
                        ++nc;
                        if (nc > (int)NCs) {
                            /* More overlapping partners than slots: the
                             * reference stops scanning this cell and drops
                             * contacts silently (contactsearch.cuh:298-299);
                             * the oracle reports it. */
                            s->capacity_hit = 1;
                            orc_set_error(s, ORC_ERR_CAPACITY,
                                          "more overlapping partners than contact slots");
                            return;
                        }
                    }
                }
            }
}

int orc_stage_topology(orc_state *s)
{
    if (s->contactmodel == 2 || s->contactmodel == 3) {
        /* each particle writes only its own slot row */
#pragma omp parallel for schedule(static)
        for (unsigned a = 0; a < s->np; ++a) topology_particle(s, a);
    }
    return s->err;
}

/* ------------------------------------------------------------------ */
/* a10: contactLinear_wall, src/contactmodels.cuh:10-114                */
/* ------------------------------------------------------------------ */
static double contact_wall(const orc_state *s, v3 *F, v3 *T, double *es_dot,
                           double *ev_dot, double *p, double ra, v3 vlin,
                           v3 angvel, v3 n, double delta, double wvel)
{
    v3 vel = adds3(add3(vlin, smul3(ra + delta / 2.0, cross3(n, angvel))), wvel);
    double vel_n = dot3(vlin, n);
    v3 vel_t = sub3(vel, muls3(n, dot3(n, vel)));
    double vel_t_length = orc_len(s, vel_t);
    double k_n = s->k_n;
    if (s->E > .001) k_n = 3.141592654 / 2.0 * s->E * ra;
    v3 f_n = smul3(fmax(0.0, -k_n * delta - s->gamma_wn * vel_n), n);
    double f_n_length = orc_len(s, f_n);
    *ev_dot += s->gamma_wn * vel_n * vel_n;
    v3 f_t = mk3(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0 && s->gamma_wt > 0.0) {
        v3 f_t_visc = smul3(s->gamma_wt, vel_t);
        double f_t_visc_length = orc_len(s, f_t_visc);
        double f_t_limit;
        if (vel_t_length > 0.0) f_t_limit = s->mu_wd * f_n_length;
        else f_t_limit = s->mu_ws * f_n_length;
        if (f_t_visc_length < f_t_limit) {
            f_t = smul3(-1.0, f_t_visc);
        } else {
            f_t = divs3(smul3(-f_t_limit, vel_t), vel_t_length);
            *es_dot += orc_len(s, muls3(smul3(orc_len(s, f_t), vel_t), s->dt)) / s->dt;
        }
    }
    *F = add3(*F, add3(f_n, f_t));
    *T = add3(*T, cross3(smul3(-(ra + delta * 0.5), n), f_t));
    *p += f_n_length / (4.0f * ORC_PI * ra * ra);
    return dot3(f_n, n);
}

/* a7: contactLinear, src/contactmodels.cuh:241-408 */
static void contact_linear(orc_state *s, v3 *F, v3 *T, double *es_dot,
                           double *ev_dot, double *p, unsigned b_orig,
                           d4 vel_a, v3 angvel_a, double ra, double rb, v3 x,
                           double x_length, double delta, size_t mempos)
{
    d4 vel_b = s->vel[b_orig];
    d4 av4b = s->angvel[b_orig];
    d4 dt0 = s->delta_t[mempos];
    v3 delta_t0_uncor = xyz(dt0);
    v3 angvel_b = xyz(av4b);
    v3 n = divs3(x, x_length);
    v3 vel_linear = mk3(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    v3 vel = add3(add3(vel_linear, smul3(ra + delta / 2.0, cross3(n, angvel_a))),
                  smul3(rb + delta / 2.0, cross3(n, angvel_b)));
    double vel_n = -dot3(vel_linear, n);
    v3 vel_t = sub3(vel, muls3(n, dot3(n, vel)));
    double vel_t_length = orc_len(s, vel_t);
    v3 delta_t0 = sub3(delta_t0_uncor, muls3(n, dot3(n, delta_t0_uncor)));
    double delta_t0_length = orc_len(s, delta_t0);
    v3 delta_t = mk3(0.0, 0.0, 0.0); /* unassigned in the reference */
    double k_n = s->k_n, k_t = s->k_t;
    if (s->E > .001) {
        k_n = 3.141592654 / 2.0 * s->E * (ra + rb) / 2.;
        k_t = k_n;
    }
    v3 f_n = smul3(fmax(0.0, -k_n * delta + s->gamma_n * vel_n), n);
    double f_n_length = orc_len(s, f_n);
    *ev_dot += 0.5 * s->gamma_n * vel_n * vel_n;
    v3 f_c = smul3(-s->kappa * orc_sqrtf(s, ra * rb), n);
    v3 f_t = mk3(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = add3(delta_t0, muls3(vel_t, s->dt));
        v3 f_t_elast = smul3(-k_t, delta_t);
        v3 f_t_visc = smul3(-s->gamma_t, vel_t);
        f_t = add3(f_t_elast, f_t_visc);
        double f_t_length = orc_len(s, f_t);
        double f_t_limit = s->mu_s * orc_len(s, sub3(f_n, f_c));
        *ev_dot += 0.5 * s->gamma_t * vel_t_length * vel_t_length;
        if (f_t_length > f_t_limit) {
            v3 t = divs3(f_t, orc_len(s, f_t));
            f_t = smul3(f_t_limit, t);
            delta_t = smul3(-1.0 / k_t,
                            add3(smul3(s->mu_d * orc_len(s, sub3(f_n, f_c)), t),
                                 smul3(s->gamma_t, vel_t)));
            *es_dot += 0.5 * orc_len(s, muls3(smul3(orc_len(s, f_t), vel_t), s->dt)) / s->dt;
        }
    }
    *F = add3(*F, add3(add3(f_n, f_t), f_c));
    *T = add3(*T, cross3(smul3(-(ra + delta * 0.5), n), f_t));
    *p += f_n_length / (4.0f * ORC_PI * ra * ra);
    d4 out = {delta_t.x, delta_t.y, delta_t.z, 0.0f};
    s->delta_t[mempos] = out;
}

/* capillaryCohesion_exp, src/cohesion.cuh:237-277 (model 1, kappa > 0) */
static void capillary_exp(const orc_state *s, v3 *N, double ra, double rb,
                          double delta_ab, v3 x_ab, double x_ab_length,
                          double kappa)
{
    v3 n_ab = divs3(x_ab, x_ab_length);
    double r;
    if ((ra / rb) > (rb / ra)) r = ra / rb;
    else r = rb / ra;
    double h = -orc_sqrtf(s, r);
    double R_har = (2.0f * ra * rb) / (ra + rb);
    double R_geo = orc_sqrtf(s, ra * rb);
    double lambda = 0.9f * h * orc_sqrtf(s, s->V_b / R_har);
    double e = s->precision == 0 ? (double)expf((float)(-delta_ab / lambda))
                                 : exp(-delta_ab / lambda);
    v3 f_c = smul3(-kappa * R_geo * e, n_ab);
    *N = add3(*N, f_c);
}

/* a8: contactLinearViscous, src/contactmodels.cuh:119-237 */
static void contact_linear_viscous(const orc_state *s, v3 *F, v3 *T, double *p,
                                   unsigned a, unsigned b, double ra, double rb,
                                   v3 x_ab, double x_ab_length, double delta_ab,
                                   double kappa)
{
    d4 vel_a = s->vel_sorted[a], vel_b = s->vel_sorted[b];
    v3 angvel_a = xyz(s->angvel_sorted[a]), angvel_b = xyz(s->angvel_sorted[b]);
    v3 n_ab = divs3(x_ab, x_ab_length);
    v3 vel_ab_linear = mk3(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    v3 vel_ab = add3(add3(vel_ab_linear,
                          smul3(ra + delta_ab / 2.0f, cross3(n_ab, angvel_a))),
                     smul3(rb + delta_ab / 2.0f, cross3(n_ab, angvel_b)));
    double vel_n_ab = dot3(vel_ab_linear, n_ab);
    v3 vel_t_ab = sub3(vel_ab, muls3(n_ab, dot3(vel_ab, n_ab)));
    double vel_t_ab_length = orc_len(s, vel_t_ab);
    double k_n = s->k_n;
    if (s->E > .001) k_n = 3.141592654 / 2.0 * s->E * (ra + rb) / 2.;
    v3 f_n = smul3(fmax(0.0, -k_n * delta_ab - s->gamma_n * vel_n_ab), n_ab);
    if (dot3(f_n, n_ab) < 0.0f) f_n = mk3(0.0f, 0.0f, 0.0f);
    double f_n_length = orc_len(s, f_n);
    v3 f_c = smul3(-kappa * orc_sqrtf(s, ra * rb), n_ab);
    v3 f_t = mk3(0.0, 0.0, 0.0);
    if (vel_t_ab_length > 0.0) {
        double f_t_visc = s->gamma_t * vel_t_ab_length;
        double f_t_limit;
        if (vel_t_ab_length > 0.001f) f_t_limit = s->mu_d * orc_len(s, sub3(f_n, f_c));
        else f_t_limit = s->mu_s * orc_len(s, sub3(f_n, f_c));
        if (f_t_visc < f_t_limit)
            f_t = divs3(smul3(-f_t_visc, vel_t_ab), vel_t_ab_length);
        else
            f_t = divs3(smul3(-f_t_limit, vel_t_ab), vel_t_ab_length);
    }
    *F = add3(*F, add3(add3(f_n, f_t), f_c));
    *T = add3(*T, smul3(-(ra + delta_ab / 2.0f), cross3(n_ab, f_t)));
    *p += f_n_length / (4.0f * ORC_PI * ra * ra);
}

/* findAndProcessContactsInCell, src/contactsearch.cuh:91-186 */
static void model1_cell(orc_state *s, int cx, int cy, int cz, unsigned a,
                        d4 xa, double ra, v3 *F, v3 *T, double *p)
{
    v3 dm = mk3(0.0f, 0.0f, 0.0f);
    if (find_distmod(s, &cx, &cy, &cz, &dm) == -1) return;
    unsigned cell = (unsigned)cx + (unsigned)cy * s->num[0] +
                    (s->num[0] * s->num[1]) * (unsigned)cz;
    unsigned start = s->cellstart[cell];
    if (start == 0xffffffffu) return;
    unsigned end = s->cellend[cell];
    for (unsigned b = start; b < end; ++b) {
        if (b == a) continue;
        d4 xb = s->x_sorted[b];
        double rb = xb.w;
        double kappa = s->kappa;
        v3 x_ab = mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
        x_ab = add3(x_ab, dm);
        double len = orc_len(s, x_ab);
        double delta_ab = len - (ra + rb);
        if (delta_ab < 0.0f)
            contact_linear_viscous(s, F, T, p, a, b, ra, rb, x_ab, len, delta_ab, kappa);
        else if (delta_ab < s->db)
            capillary_exp(s, F, ra, rb, delta_ab, x_ab, len, kappa);
    }
}

/* a6 + a10 + a11: interact, src/contactsearch.cuh:385-726 */
static void interact_particle(orc_state *s, unsigned a)
{
    unsigned a_orig = s->index[a];
    d4 xa = s->x_sorted[a];
    double ra = xa.w;
    v3 origo = mk3(s->origo[0], s->origo[1], s->origo[2]);
    v3 L = mk3(s->L[0], s->L[1], s->L[2]);
    d4 wnx[5] = {{0.0f, 0.0f, -1.0f, L.z}, {-1.0f, 0.0f, 0.0f, L.x},
                 {1.0f, 0.0f, 0.0f, 0.0f}, {0.0f, -1.0f, 0.0f, L.y},
                 {0.0f, 1.0f, 0.0f, 0.0f}};
    d4 wmvfd[5] = {{0}, {0}, {0}, {0}, {0}};
    for (unsigned w = 0; w < s->nw && w < 5; ++w) {
        wnx[w] = s->wnx[w];
        wmvfd[w] = s->wmvfd[w];
    }
    double es_dot = 0.0, ev_dot = 0.0, p = 0.0;
    v3 F = mk3(0.0, 0.0, 0.0), T = mk3(0.0, 0.0, 0.0);
    d4 vel_a = s->vel_sorted[a];
    v3 angvel_a = xyz(s->angvel_sorted[a]);
    if (s->contactmodel == 2 || s->contactmodel == 3) {
        for (unsigned i = 0; i < s->nc; ++i) {
            size_t mempos = (size_t)a_orig * s->nc + i;
            unsigned b_orig = s->contacts[mempos];
            if (b_orig != s->np) {
                d4 dm = s->distmod[mempos];
                d4 xb = s->x[b_orig];
                double rb = xb.w;
                v3 x_ab = mk3(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
                double len = orc_len(s, x_ab);
                double delta_n = len - (ra + rb);
                if (delta_n < 0.0) {
                    contact_linear(s, &F, &T, &es_dot, &ev_dot, &p, b_orig, vel_a,
                                   angvel_a, ra, rb, x_ab, len, delta_n, mempos);
                } else {
                    s->contacts[mempos] = s->np;
                    d4 z = {0.0, 0.0, 0.0, 0.0};
                    s->delta_t[mempos] = z;
                }
            } else {
                d4 z = {0.0, 0.0, 0.0, 0.0};
                s->delta_t[mempos] = z;
            }
        }
    } else if (s->contactmodel == 1) {
        int gx, gy, gz;
        grid_pos(s, xa, &gx, &gy, &gz);
        for (int dz = -1; dz < 2; ++dz)
            for (int dy = -1; dy < 2; ++dy)
                for (int dx = -1; dx < 2; ++dx)
                    model1_cell(s, gx + dx, gy + dy, gz + dz, a, xa, ra, &F, &T, &p);
    }

    double wf[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    v3 vlin = xyz(vel_a);
    double dw;
    dw = wnx[0].w - (xa.z + ra);
    if (dw < 0.0f)
        wf[0] = contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                             xyz(wnx[0]), dw, wmvfd[0].y);
    dw = xa.z - ra - origo.z;
    if (dw < 0.0f)
        (void)contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                           mk3(0.0f, 0.0f, 1.0f), dw, 0.0);
    if (s->periodic == 0) {
        dw = wnx[1].w - (xa.x + ra);
        if (dw < 0.0f)
            wf[1] = contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                                 xyz(wnx[1]), dw, wmvfd[1].y);
        dw = xa.x - ra - wnx[2].w;
        if (dw < 0.0f)
            wf[2] = contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                                 xyz(wnx[2]), dw, wmvfd[2].y);
    }
    if (s->periodic == 0 || s->periodic == 2) {
        dw = wnx[3].w - (xa.y + ra);
        if (dw < 0.0f)
            wf[3] = contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                                 xyz(wnx[3]), dw, wmvfd[3].y);
        dw = xa.y - ra - wnx[4].w;
        if (dw < 0.0f)
            wf[4] = contact_wall(s, &F, &T, &es_dot, &ev_dot, &p, ra, vlin, angvel_a,
                                 xyz(wnx[4]), dw, wmvfd[4].y);
    }
    d4 f4 = {F.x, F.y, F.z, 0.0f}, t4 = {T.x, T.y, T.z, 0.0f};
    s->force[a_orig] = f4;
    s->torque[a_orig] = t4;
    s->es_dot[a_orig] = es_dot;
    s->ev_dot[a_orig] = ev_dot;
    s->es[a_orig] += es_dot * s->dt;
    s->ev[a_orig] += ev_dot * s->dt;
    s->p[a_orig] = p;
    for (unsigned w = 0; w < s->nw && w < 5; ++w)
        s->walls_force_pp[a_orig + (size_t)s->np * w] = wf[w];
}

int orc_stage_interact(orc_state *s)
{
    if (s->contactmodel == 3) {
        orc_set_error(s, ORC_ERR_UNSUPPORTED, "contact model 3 (Hertz) is not built");
        return s->err;
    }
    /* each particle writes only its own row and its own outputs */
#pragma omp parallel for schedule(static)
    for (unsigned a = 0; a < s->np; ++a) interact_particle(s, a);
    return s->err;
}

/* ------------------------------------------------------------------ */
/* a14: summation, src/integration.cuh:309-341 (256-wide tree per block) */
/* ------------------------------------------------------------------ */
void orc_block_sums(const double *in, unsigned n, double *out, unsigned nblocks)
{
    double cache[256];
    for (unsigned b = 0; b < nblocks; ++b) {
        for (unsigned t = 0; t < 256; ++t) {
            unsigned idx = b * 256 + t;
            double temp = 0.0f;
            while (idx < n) {
                temp += in[idx];
                idx += 256 * nblocks;
            }
            cache[t] = temp;
        }
        for (unsigned i = 128; i != 0; i /= 2)
            for (unsigned t = 0; t < i; ++t) cache[t] += cache[t + i];
        out[b] = cache[0];
    }
}

/* a15: findShearStressOnFixedMovingParticles, integration.cuh:457-484 */
static void stage_shear_stress(orc_state *s)
{
    for (unsigned i = 0; i < s->np; ++i) {
        double z = s->x[i].z, fixvel = s->vel[i].w, fx = s->force[i].x;
        double f_x = 0.0;
        if (fixvel > 0.0 && z > s->L[2] * 0.5) f_x = fx;
        s->tau_eff_pp[i] = f_x / (s->L[0] * s->L[1]);
    }
    orc_block_sums(s->tau_eff_pp, s->np, s->tau_partials, s->nblocks);
}

/* a13: integrate, src/integration.cuh:14-305 */
static void integrate_particle(orc_state *s, unsigned i, int change_velocity_state,
                               double velocity_factor)
{
    unsigned o = s->index[i];
    d4 force = s->force[o], torque = s->torque[o], angpos = s->angpos[o];
    d4 x = s->x_sorted[i], vel = s->vel_sorted[i], angvel = s->angvel_sorted[i];
    d4 xyzsum = s->xyzsum[o];
    int wall0mode = 0;
    double wall0mass = 0.0;
    if (s->nw > 0) {
        wall0mode = s->wmode[0];
        wall0mass = s->wmvfd[0].x;
    }
    double tau_eff_x = 0.0;
    if (s->nw > 0 && wall0mode == 3)
        for (unsigned b = 0; b < s->nblocks; ++b) tau_eff_x += s->tau_partials[b];
    d4 acc0 = {0, 0, 0, 0}, angacc0 = {0, 0, 0, 0};
    if (s->iter != 0) {
        acc0 = s->acc[o];
        angacc0 = s->angacc[o];
    }
    double radius = x.w;
    double dt = s->dt;
    double m = 4.0 / 3.0 * ORC_PI * radius * radius * radius * s->rho;
    d4 acc = {0.0, 0.0, 0.0, 0.0};
    acc.x = force.x / m + s->g[0];
    acc.y = force.y / m + s->g[1];
    acc.z = force.z / m + s->g[2];
    d4 angacc = {0.0, 0.0, 0.0, 0.0};
    angacc.x = torque.x * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc.y = torque.y * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc.z = torque.z * 1.0 / (2.0 / 5.0 * m * radius * radius);
    d4 zero4 = {0.0, 0.0, 0.0, 0.0};
    if (wall0mode == 3 && vel.w > 0.0001 && x.z > s->L[2] * 0.5) {
        double f_tau_x = (s->tau_x + tau_eff_x) * s->L[0] * s->L[1];
        acc.x = f_tau_x / wall0mass;
        acc.y = 0.0;
        acc.z -= s->g[2];
        angacc = zero4;
    } else if (vel.w > 0.0001 && vel.w < 10.0) {
        acc.x = 0.0;
        acc.y = 0.0;
        acc.z -= s->g[2];
        angacc = zero4;
    }
    if (vel.w >= 10.0) {
        acc.y = 0.0;
        angacc.x = 0.0;
        angacc.z = 0.0;
    }
    if (vel.w < -0.0001) {
        acc.x = 0.0;
        acc.y = 0.0;
        acc.z = 0.0;
        angacc = zero4;
    }
    d4 x_new, vel_new, angpos_new, angvel_new;
    if (s->integrator == 3) {
        double dax = (acc.x - acc0.x) / dt, day = (acc.y - acc0.y) / dt,
               daz = (acc.z - acc0.z) / dt;
        double dwx = (angacc.x - angacc0.x) / dt, dwy = (angacc.y - angacc0.y) / dt,
               dwz = (angacc.z - angacc0.z) / dt;
        x_new.x = x.x + vel.x * dt + 0.5 * acc.x * dt * dt + 1.0 / 6.0 * dax * dt * dt * dt;
        x_new.y = x.y + vel.y * dt + 0.5 * acc.y * dt * dt + 1.0 / 6.0 * day * dt * dt * dt;
        x_new.z = x.z + vel.z * dt + 0.5 * acc.z * dt * dt + 1.0 / 6.0 * daz * dt * dt * dt;
        x_new.w = x.w;
        vel_new.x = vel.x + acc.x * dt + 0.5 * dax * dt * dt;
        vel_new.y = vel.y + acc.y * dt + 0.5 * day * dt * dt;
        vel_new.z = vel.z + acc.z * dt + 0.5 * daz * dt * dt;
        vel_new.w = vel.w;
        angpos_new.x = angpos.x + angvel.x * dt + 0.5 * angacc.x * dt * dt
                       + 1.0 / 6.0 * dwx * dt * dt * dt;
        angpos_new.y = angpos.y + angvel.y * dt + 0.5 * angacc.y * dt * dt
                       + 1.0 / 6.0 * dwy * dt * dt * dt;
        angpos_new.z = angpos.z + angvel.z * dt + 0.5 * angacc.z * dt * dt
                       + 1.0 / 6.0 * dwz * dt * dt * dt;
        angpos_new.w = angpos.w;
        angvel_new.x = angvel.x + angacc.x * dt + 0.5 * dwx * dt * dt;
        angvel_new.y = angvel.y + angacc.y * dt + 0.5 * dwy * dt * dt;
        angvel_new.z = angvel.z + angacc.z * dt + 0.5 * dwz * dt * dt;
        angvel_new.w = angvel.w;
        xyzsum.x += vel.x * dt + 0.5 * acc.x * dt * dt + 1.0 / 6.0 * dax * dt * dt * dt;
        xyzsum.y += vel.y * dt + 0.5 * acc.y * dt * dt + 1.0 / 6.0 * day * dt * dt * dt;
        xyzsum.z += vel.z * dt + 0.5 * acc.z * dt * dt + 1.0 / 6.0 * daz * dt * dt * dt;
    } else {
        /* TY2, integration.cuh:192-220 */
        x_new.x = x.x + vel.x * dt + 0.5 * acc.x * dt * dt;
        x_new.y = x.y + vel.y * dt + 0.5 * acc.y * dt * dt;
        x_new.z = x.z + vel.z * dt + 0.5 * acc.z * dt * dt;
        x_new.w = x.w;
        vel_new.x = vel.x + acc.x * dt;
        vel_new.y = vel.y + acc.y * dt;
        vel_new.z = vel.z + acc.z * dt;
        vel_new.w = vel.w;
        angpos_new.x = angpos.x + angvel.x * dt + 0.5 * angacc.x * dt * dt;
        angpos_new.y = angpos.y + angvel.y * dt + 0.5 * angacc.y * dt * dt;
        angpos_new.z = angpos.z + angvel.z * dt + 0.5 * angacc.z * dt * dt;
        angpos_new.w = angpos.w;
        angvel_new.x = angvel.x + angacc.x * dt;
        angvel_new.y = angvel.y + angacc.y * dt;
        angvel_new.z = angvel.z + angacc.z * dt;
        angvel_new.w = angvel.w;
        xyzsum.x += vel.x * dt + 0.5 * acc.x * dt * dt;
        xyzsum.y += vel.y * dt + 0.5 * acc.y * dt * dt;
        xyzsum.z += vel.z * dt + 0.5 * acc.z * dt * dt;
    }
    if (s->periodic == 1) {
        if (x_new.x < s->origo[0]) x_new.x += s->L[0];
        if (x_new.x > s->L[0]) x_new.x -= s->L[0];
        if (x_new.y < s->origo[1]) x_new.y += s->L[1];
        if (x_new.y > s->L[1]) x_new.y -= s->L[1];
    } else if (s->periodic == 2) {
        if (x_new.x < s->origo[0]) x_new.x += s->L[0];
        if (x_new.x > s->L[0]) x_new.x -= s->L[0];
    }
    if (vel.w > 5.0 && vel.w < 10.0) {
        if (change_velocity_state == 1) vel_new.x *= velocity_factor;
        else if (change_velocity_state == -1) vel_new.x /= velocity_factor;
    }
    s->xyzsum[o] = xyzsum;
    s->acc[o] = acc;
    s->angacc[o] = angacc;
    s->angvel[o] = angvel_new;
    s->vel[o] = vel_new;
    s->angpos[o] = angpos_new;
    s->x[o] = x_new;
}

/* integrateWalls, src/integration.cuh:344-450 */
static void integrate_walls(orc_state *s)
{
    for (unsigned w = 0; w < s->nw; ++w) {
        d4 w_nx = s->wnx[w], w_mvfd = s->wmvfd[w];
        int wmode = s->wmode[w];
        if (wmode == 0) continue;
        double acc0 = s->iter == 0 ? 0.0 : s->w_acc[w];
        w_mvfd.z = 0.0;
        for (unsigned b = 0; b < s->nblocks; ++b) w_mvfd.z += s->force_partials[b];
        double dt = s->dt;
        double sigma_0 = w_mvfd.w + s->sigma0_A * sin(2.0 * ORC_PI * s->sigma0_f * s->t_current);
        double N = -sigma_0 * s->L[0] * s->L[1];
        double acc = (w_mvfd.z + N) / w_mvfd.x;
        if (wmode == 2) acc = 0.0;
        if (s->integrator == 3) {
            double dacc_dt = (acc - acc0) / dt;
            w_nx.w += w_mvfd.y * dt + 0.5 * acc * dt * dt + 1.0 / 6.0 * dacc_dt * dt * dt * dt;
            w_mvfd.y += acc * dt + 0.5 * dacc_dt * dt * dt;
        } else {
            w_nx.w += w_mvfd.y * dt + 0.5 * acc * dt * dt;
            w_mvfd.y += acc * dt;
        }
        s->wnx[w] = w_nx;
        s->wmvfd[w] = w_mvfd;
        s->w_acc[w] = acc;
    }
}

/* One iteration of the time loop, device.cu:1038-2550 (dry part) */
static int one_step(orc_state *s)
{
    if (s->np > 0) {
        int rc = orc_stage_hash_sort_reorder(s);
        if (rc) return rc;
        if ((rc = orc_stage_topology(s))) return rc;
        if ((rc = orc_stage_interact(s))) return rc;
        if (s->nb0 > 0) orc_bonds(s);
    }
    if (s->fluid && s->cfd_solver == 1) {
        int rc = orc_darcy_step(s);
        if (rc && rc != ORC_ERR_NOCONV) return rc;
    }
    if (s->np > 0) {
        if (s->nw > 0 && s->wmode[0] == 3) stage_shear_stress(s);
        /* rate-state velocity step, device.cu:1000-1005,2461-2469 */
        int change = 0;
        const double velocity_factor = 10.0, v2_start = 10.0, v2_end = 15.0;
        if (s->t_current >= v2_start && s->t_current < v2_end && s->velocity_state == 1) {
            change = 1;
            s->velocity_state = 2;
        } else if (s->t_current >= v2_end && s->velocity_state == 2) {
            change = -1;
            s->velocity_state = 1;
        }
#pragma omp parallel for schedule(static)
        for (unsigned i = 0; i < s->np; ++i) integrate_particle(s, i, change, velocity_factor);
        if (s->nw > 0) {
            orc_block_sums(s->walls_force_pp, s->np, s->force_partials, s->nblocks);
            integrate_walls(s);
        }
    }
    s->t_current += s->dt;
    s->filetimeclock += s->dt;
    s->iter++;
    return s->err;
}

int orc_step(orc_state *s, int64_t nsteps)
{
    for (int64_t k = 0; k < nsteps; ++k) {
        int rc = one_step(s);
        if (rc) return rc;
    }
    return s->err;
}

const char *orc_error(const orc_state *s) { return s ? s->errmsg : "no state"; }
int orc_np(const orc_state *s) { return (int)s->np; }
int orc_nc(const orc_state *s) { return (int)s->nc; }
int orc_nw(const orc_state *s) { return (int)s->nw; }
