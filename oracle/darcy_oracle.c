/*
 * Darcy pressure solver for the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 * Restates the cfd_solver == 1 block of DEM::startTime
 * (src/device.cu:1901-2426) and its kernels (src/darcy.cuh), serially.
 * Fields are ghost-padded (nx+2)(ny+2)(nz+2) as in the reference
 * (src/darcy.cpp:36-40); ghost cells start at zero.
 */
#include "sph_oracle.h"
#include "oracle_internal.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct orc_darcy {
    int nx, ny, nz;
    size_t ng;
    double *p, *p_new, *p_old, *dp_expl, *phi, *dphi, *k, *norm, *div_v_p;
    double *v, *vp_avg, *grad_p, *grad_k; /* 3 per cell */
    int *p_constant;
    d4 *f_p;
    double mu, rho_f, p_mod_A, p_mod_f, p_mod_phi;
    int bc_xn, bc_xp, bc_yn, bc_yp, bc_bot, bc_top, free_slip_bot, free_slip_top;
    double bc_bot_flux, bc_top_flux, tolerance, c_phi, beta_f, k_c;
    unsigned maxiter, ndem;
    double p_top_orig;
    unsigned wall0_iz;
    int64_t nijac_last, nijac_total;
    int exact_stop; /* test the residual every iteration (the engine's option);
                       0: at iterations 0, 10, 20, ... as device.cu:2340-2366 */
};

/* d_idx, src/darcy.cuh:128-137 (unsigned arithmetic like the reference) */
static inline unsigned didx(const struct orc_darcy *D, int x, int y, int z)
{
    return (unsigned)(x + 1) + ((unsigned)D->nx + 2u) * (unsigned)(y + 1) +
           ((unsigned)D->nx + 2u) * ((unsigned)D->ny + 2u) * (unsigned)(z + 1);
}

static void *zalloc(size_t n, size_t sz)
{
    void *p = calloc(n ? n : 1, sz);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

typedef struct { const unsigned char *p, *end; int bad; } rd;
static void take(rd *r, void *dst, size_t n)
{
    if (r->bad || (size_t)(r->end - r->p) < n) { r->bad = 1; memset(dst, 0, n); return; }
    memcpy(dst, r->p, n);
    r->p += n;
}
static double rf8(rd *r) { double v; take(r, &v, 8); return v; }
static unsigned ru4(rd *r) { unsigned v; take(r, &v, 4); return v; }
static int ri4(rd *r) { int v; take(r, &v, 4); return v; }

int orc_darcy_load(orc_state *s, const unsigned char **cur, const unsigned char *end)
{
    struct orc_darcy *D = (struct orc_darcy *)zalloc(1, sizeof *D);
    s->darcy = D;
    D->nx = (int)s->num[0];
    D->ny = (int)s->num[1];
    D->nz = (int)s->num[2];
    D->ng = (size_t)(D->nx + 2) * (D->ny + 2) * (D->nz + 2);
    size_t ng = D->ng;
    D->p = zalloc(ng, 8); D->p_new = zalloc(ng, 8); D->p_old = zalloc(ng, 8);
    D->dp_expl = zalloc(ng, 8); D->phi = zalloc(ng, 8); D->dphi = zalloc(ng, 8);
    D->k = zalloc(ng, 8); D->norm = zalloc(ng, 8); D->div_v_p = zalloc(ng, 8);
    D->v = zalloc(3 * ng, 8); D->vp_avg = zalloc(3 * ng, 8);
    D->grad_p = zalloc(3 * ng, 8); D->grad_k = zalloc(3 * ng, 8);
    D->p_constant = zalloc(ng, sizeof(int));
    D->f_p = zalloc(s->np, sizeof(d4));
    D->wall0_iz = 10000000u;
    rd r = {*cur, end, 0};
    D->mu = rf8(&r);
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) {
                unsigned i = didx(D, x, y, z);
                take(&r, &D->v[3 * (size_t)i], 24);
                D->p[i] = rf8(&r);
                D->phi[i] = rf8(&r);
                D->dphi[i] = rf8(&r);
            }
    D->rho_f = rf8(&r); D->p_mod_A = rf8(&r); D->p_mod_f = rf8(&r); D->p_mod_phi = rf8(&r);
    D->bc_xn = ri4(&r); D->bc_xp = ri4(&r); D->bc_yn = ri4(&r); D->bc_yp = ri4(&r);
    D->bc_bot = ri4(&r); D->bc_top = ri4(&r);
    D->free_slip_bot = ri4(&r); D->free_slip_top = ri4(&r);
    D->bc_bot_flux = rf8(&r); D->bc_top_flux = rf8(&r);
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) D->p_constant[didx(D, x, y, z)] = ri4(&r);
    D->tolerance = rf8(&r); D->maxiter = ru4(&r); D->ndem = ru4(&r); D->c_phi = rf8(&r);
    for (unsigned i = 0; i < s->np; ++i) take(&r, &D->f_p[i], 24);
    D->beta_f = rf8(&r); D->k_c = rf8(&r);
    if (r.bad) return ORC_ERR_INPUT;
    if (D->ndem == 0) return ORC_ERR_INPUT;
    /* device.cu:1017-1020 */
    D->p_top_orig = D->p[didx(D, 0, 0, D->nz - 1)] -
                    D->p_mod_A * sin(2.0 * M_PI * D->p_mod_f * s->t_current + D->p_mod_phi);
    s->host_wall0_w = s->nw > 0 ? s->wnx[0].w : 0.0;
    *cur = r.p;
    return 0;
}

void orc_darcy_free(orc_state *s)
{
    struct orc_darcy *D = s->darcy;
    if (!D) return;
    free(D->p); free(D->p_new); free(D->p_old); free(D->dp_expl); free(D->phi);
    free(D->dphi); free(D->k); free(D->norm); free(D->div_v_p); free(D->v);
    free(D->vp_avg); free(D->grad_p); free(D->grad_k); free(D->p_constant); free(D->f_p);
    free(D);
    s->darcy = NULL;
}

int orc_darcy_write(orc_state *s, void *fh)
{
    struct orc_darcy *D = s->darcy;
    FILE *f = (FILE *)fh;
    fwrite(&D->mu, 8, 1, f);
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) {
                unsigned i = didx(D, x, y, z);
                fwrite(&D->v[3 * (size_t)i], 8, 3, f);
                fwrite(&D->p[i], 8, 1, f);
                fwrite(&D->phi[i], 8, 1, f);
                fwrite(&D->dphi[i], 8, 1, f);
            }
    double a[] = {D->rho_f, D->p_mod_A, D->p_mod_f, D->p_mod_phi};
    fwrite(a, 8, 4, f);
    int b[] = {D->bc_xn, D->bc_xp, D->bc_yn, D->bc_yp, D->bc_bot, D->bc_top,
               D->free_slip_bot, D->free_slip_top};
    fwrite(b, 4, 8, f);
    fwrite(&D->bc_bot_flux, 8, 1, f);
    fwrite(&D->bc_top_flux, 8, 1, f);
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) fwrite(&D->p_constant[didx(D, x, y, z)], 4, 1, f);
    fwrite(&D->tolerance, 8, 1, f);
    fwrite(&D->maxiter, 4, 1, f);
    fwrite(&D->ndem, 4, 1, f);
    fwrite(&D->c_phi, 8, 1, f);
    for (unsigned i = 0; i < s->np; ++i) fwrite(&D->f_p[i], 8, 3, f);
    fwrite(&D->beta_f, 8, 1, f);
    fwrite(&D->k_c, 8, 1, f);
    return 0;
}

/* setDarcyGhostNodes<T>, darcy.cuh:194-264 (comps doubles per cell) */
static void ghost(const orc_state *s, struct orc_darcy *D, double *f, int comps)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    (void)s;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double *val = &f[(size_t)comps * didx(D, x, y, z)];
#define PUT(X, Y, Z) memcpy(&f[(size_t)comps * didx(D, X, Y, Z)], val, 8 * (size_t)comps)
                if (x == 0 && D->bc_xn == 0) PUT(-1, y, z);
                if (x == 1 && D->bc_xn == 1) PUT(-1, y, z);
                if (x == 0 && D->bc_xn == 2) PUT(nx, y, z);
                if (x == nx - 1 && D->bc_xp == 0) PUT(nx, y, z);
                if (x == nx - 2 && D->bc_xp == 1) PUT(nx, y, z);
                if (x == nx - 1 && D->bc_xp == 2) PUT(-1, y, z);
                if (y == 0 && D->bc_yn == 0) PUT(x, -1, z);
                if (y == 1 && D->bc_yn == 1) PUT(x, -1, z);
                if (y == 0 && D->bc_yn == 2) PUT(x, ny, z);
                if (y == ny - 1 && D->bc_yp == 0) PUT(x, ny, z);
                if (y == ny - 2 && D->bc_yp == 1) PUT(x, ny, z);
                if (y == ny - 1 && D->bc_yp == 2) PUT(x, -1, z);
                if (z == 0 && D->bc_bot == 0) PUT(x, y, -1);
                if (z == 1 && D->bc_bot == 1) PUT(x, y, -1);
                if (z == 0 && D->bc_bot == 2) PUT(x, y, nz);
                if (z == nz - 1 && D->bc_top == 0) PUT(x, y, nz);
                if (z == nz - 2 && D->bc_top == 1) PUT(x, y, nz);
                if (z == nz - 1 && D->bc_top == 2) PUT(x, y, -1);
#undef PUT
            }
}

/* setDarcyGhostNodesFlux, darcy.cuh:270-312 */
static void ghost_flux(const orc_state *s, struct orc_darcy *D)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double p = D->p[didx(D, x, y, z)];
                double k = D->k[didx(D, x, y, z)];
                double dz = s->L[2] / nz;
                double q_z = 0.;
                if (z == 0) q_z = D->bc_bot_flux;
                else if (z == nz - 1) q_z = D->bc_top_flux;
                double p_ghost = -D->mu / k * q_z * dz + p;
                if (z == 0 && D->bc_bot == 4) D->p[didx(D, x, y, -1)] = p_ghost;
                if (z == nz - 1 && D->bc_top == 4) D->p[didx(D, x, y, nz)] = p_ghost;
            }
}

/* The reference's pow calls.  Built with ORC_POW_AS_PRODUCTS (the
 * liboracle_powprod.so variant) they become products, which differ from
 * pow in the last bit: a probe of how far last-bit differences of a math
 * library (CUDA's pow on the device against glibc's here) move the solve. */
#ifdef ORC_POW_AS_PRODUCTS
#define ORC_CUBE(v) ((v) * (v) * (v))
#define ORC_SQUARE(v) ((v) * (v))
#else
#define ORC_CUBE(v) pow((v), 3)
#define ORC_SQUARE(v) pow((v), 2)
#endif

static inline double sphere_volume(double r) { return 4.0 / 3.0 * M_PI * ORC_CUBE(r); }

static double weight_dist(v3 d, double dx, double dy, double dz)
{
    v3 a = {fabs(d.x), fabs(d.y), fabs(d.z)};
    if (a.x < dx && a.y < dy && a.z < dz)
        return (1.0 - a.x / dx) * (1.0 - a.y / dy) * (1.0 - a.z / dz);
    return 0.0;
}

/* findDistMod for the porosity kernel (contactsearch.cuh:12-83) */
static int dm_cell(const orc_state *s, int *cx, int *cy, int *cz, v3 *dm)
{
    int nx = (int)s->num[0], ny = (int)s->num[1], nz = (int)s->num[2];
    if (s->periodic == 1) {
        if (*cx < 0) { *cx += nx; dm->x = dm->x + s->L[0]; dm->y = dm->y + 0.0; dm->z = dm->z + 0.0; }
        if (*cx >= nx) { *cx -= nx; dm->x = dm->x - s->L[0]; dm->y = dm->y - 0.0; dm->z = dm->z - 0.0; }
        if (*cy < 0) { *cy += ny; dm->x = dm->x + 0.0; dm->y = dm->y + s->L[1]; dm->z = dm->z + 0.0; }
        if (*cy >= ny) { *cy -= ny; dm->x = dm->x - 0.0; dm->y = dm->y - s->L[1]; dm->z = dm->z - 0.0; }
    }
    if (s->periodic == 2) {
        if (*cx < 0) { *cx += nx; dm->x = dm->x + s->L[0]; dm->y = dm->y + 0.0; dm->z = dm->z + 0.0; }
        if (*cx >= nx) { *cx -= nx; dm->x = dm->x - s->L[0]; dm->y = dm->y - 0.0; dm->z = dm->z - 0.0; }
        if (*cy < 0 || *cy >= ny) return -1;
    }
    if (s->periodic > 2 || s->periodic < 1) {
        if (*cx < 0 || *cx >= nx) return -1;
        if (*cy < 0 || *cy >= ny) return -1;
    }
    if (*cz < 0 || *cz >= nz) return -1;
    return 0;
}

/* findDarcyPorositiesLinear, darcy.cuh:359-550 */
static void porosities(orc_state *s, struct orc_darcy *D)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                unsigned cellidx = didx(D, x, y, z);
                if (s->np == 0) {
                    D->phi[cellidx] = 0.9;
                    D->dphi[cellidx] = 0.0;
                    continue;
                }
                v3 X = {x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz};
                double solid = 0.0, solid_new = 0.0;
                v3 num = {0.0, 0.0, 0.0};
                double den = 0.0;
                double phi_0 = D->phi[cellidx];
                for (int dzc = -1; dzc < 2; ++dzc)
                    for (int dyc = -1; dyc < 2; ++dyc)
                        for (int dxc = -1; dxc < 2; ++dxc) {
                            int cx = x + dxc, cy = y + dyc, cz = z + dzc;
                            if (cz == -1) cz = 1;
                            if (s->periodic == 2) {
                                if (cy == -1) cy = 1;
                                if (cy == (int)s->num[1]) cy = (int)s->num[1] - 2;
                            }
                            v3 dm = {0.0, 0.0, 0.0};
                            if (dm_cell(s, &cx, &cy, &cz, &dm) == -1) continue;
                            unsigned cell = (unsigned)cx + (unsigned)cy * s->num[0] +
                                            (s->num[0] * s->num[1]) * (unsigned)cz;
                            unsigned start = s->cellstart[cell];
                            if (start == 0xffffffffu) continue;
                            unsigned end = s->cellend[cell];
                            for (unsigned i = start; i < end; ++i) {
                                d4 xr = s->x_sorted[i], v = s->vel_sorted[i];
                                v3 dist = {X.x - xr.x, X.y - xr.y, X.z - xr.z};
                                dist.x = dist.x + dm.x; dist.y = dist.y + dm.y; dist.z = dist.z + dm.z;
                                double sw = weight_dist(dist, dx, dy, dz);
                                double vol_p = sphere_volume(xr.w);
                                solid += sw * vol_p;
                                double sv = sw * vol_p;
                                num.x += sv * v.x; num.y += sv * v.y; num.z += sv * v.z;
                                den += sw * vol_p;
                                xr.x += v.x * s->dt; xr.y += v.y * s->dt; xr.z += v.z * s->dt;
                                v3 d2 = {X.x - xr.x, X.y - xr.y, X.z - xr.z};
                                d2.x = d2.x + dm.x; d2.y = d2.y + dm.y; d2.z = d2.z + dm.z;
                                solid_new += weight_dist(d2, dx, dy, dz) * vol_p;
                            }
                        }
                double cell_volume = dx * dy * dz;
                if (z == nz - 1) cell_volume *= 0.875;
                double phi = fmin(0.9, fmax(0.1, 1.0 - solid / cell_volume));
                double phi_new = fmin(0.9, fmax(0.1, 1.0 - solid_new / cell_volume));
                double dphi;
                v3 vp = {0.0, 0.0, 0.0};
                if (s->iter == 0) {
                    dphi = 0.0;
                } else {
                    dphi = 0.5 * (phi_new - phi_0);
                    double dd = fmax(1.0e-16, den);
                    vp.x = num.x / dd; vp.y = num.y / dd; vp.z = num.z / dd;
                }
                D->phi[cellidx] = phi * D->c_phi;
                D->dphi[cellidx] = dphi * D->c_phi;
                D->vp_avg[3 * (size_t)cellidx] = vp.x;
                D->vp_avg[3 * (size_t)cellidx + 1] = vp.y;
                D->vp_avg[3 * (size_t)cellidx + 2] = vp.z;
            }
}

/* copyDarcyPorositiesToEdges / ToBottom, darcy.cuh:556-628 */
static void copy_edges(orc_state *s, struct orc_darcy *D)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    (void)s;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                if (!(y == 0 || y == ny - 1)) continue;
                int yr = y == 0 ? 1 : ny - 2;
                unsigned r = didx(D, x, yr, z), w = didx(D, x, y, z);
                D->phi[w] = D->phi[r];
                D->dphi[w] = D->dphi[r];
                D->div_v_p[w] = D->div_v_p[r];
                memcpy(&D->vp_avg[3 * (size_t)w], &D->vp_avg[3 * (size_t)r], 24);
            }
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            unsigned r = didx(D, x, y, 1), w = didx(D, x, y, 0);
            D->phi[w] = D->phi[r];
            D->dphi[w] = D->dphi[r];
            D->div_v_p[w] = D->div_v_p[r];
            memcpy(&D->vp_avg[3 * (size_t)w], &D->vp_avg[3 * (size_t)r], 24);
        }
}

/* findDarcyPressureGradient, darcy.cuh:889-943 */
static void pressure_gradient(const orc_state *s, struct orc_darcy *D)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double *g = &D->grad_p[3 * (size_t)didx(D, x, y, z)];
                g[0] = (D->p[didx(D, x + 1, y, z)] - D->p[didx(D, x - 1, y, z)]) / (dx + dx);
                g[1] = (D->p[didx(D, x, y + 1, z)] - D->p[didx(D, x, y - 1, z)]) / (dy + dy);
                g[2] = (D->p[didx(D, x, y, z + 1)] - D->p[didx(D, x, y, z - 1)]) / (dz + dz);
            }
}

/* findDarcyPressureForceLinear, darcy.cuh:948-1102 */
static void pressure_force(orc_state *s, struct orc_darcy *D)
{
    const unsigned nx = (unsigned)D->nx, ny = (unsigned)D->ny, nz = (unsigned)D->nz;
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    const unsigned wall0_iz = D->wall0_iz;
    for (unsigned i = 0; i < s->np; ++i) {
        d4 x = s->x[i];
        unsigned i_x = (unsigned)floor((x.x - s->origo[0]) / (s->L[0] / s->num[0]));
        unsigned i_y = (unsigned)floor((x.y - s->origo[1]) / (s->L[1] / s->num[1]));
        unsigned i_z = (unsigned)floor((x.z - s->origo[2]) / (s->L[2] / s->num[2]));
        v3 X = {i_x * dx + 0.5 * dx, i_y * dy + 0.5 * dy, i_z * dz + 0.5 * dz};
        v3 gp = {0., 0., 0.};
        for (int d_iz = -1; d_iz < 2; d_iz++)
            for (int d_iy = -1; d_iy < 2; d_iy++)
                for (int d_ix = -1; d_ix < 2; d_ix++) {
                    int ix_n = (int)i_x + d_ix, iy_n = (int)i_y + d_iy, iz_n = (int)i_z + d_iz;
                    const double *gs = &D->grad_p[3 * (size_t)didx(D, ix_n, iy_n, iz_n)];
                    v3 g = {gs[0], gs[1], gs[2]};
                    if ((ix_n == -1 && iy_n == -1) || (ix_n == -1 && iz_n == -1) ||
                        (iy_n == -1 && iz_n == -1) || (ix_n == (int)nx && iy_n == (int)ny) ||
                        (ix_n == (int)nx && iz_n == (int)nz) || (iy_n == (int)ny && iz_n == (int)nz) ||
                        (ix_n == (int)nx && iy_n == -1) || (ix_n == (int)nx && iz_n == -1) ||
                        (iy_n == (int)ny && ix_n == -1) || (iy_n == (int)ny && iz_n == -1) ||
                        (iz_n == (int)nz && ix_n == -1) || (iz_n == (int)nz && iy_n == -1)) {
                        g.x = 0.; g.y = 0.; g.z = 0.;
                    }
                    /* unsigned comparison, as in the reference */
                    if (D->bc_top == 0 && i_z + (unsigned)d_iz >= wall0_iz - 1u) g.z = 0.0;
                    v3 n = {dx * d_ix, dy * d_iy, dz * d_iz};
                    v3 xf = {X.x + n.x, X.y + n.y, X.z + n.z};
                    v3 dd = {x.x - xf.x, x.y - xf.y, x.z - xf.z};
                    double w = weight_dist(dd, dx, dy, dz);
                    gp.x += w * g.x; gp.y += w * g.y; gp.z += w * g.z;
                }
        double v = sphere_volume(x.w);
        v3 f_p;
        {
            double rv = D->rho_f * v;
            f_p.x = (-1.0 * gp.x) * v - rv * s->g[0];
            f_p.y = (-1.0 * gp.y) * v - rv * s->g[1];
            f_p.z = (-1.0 * gp.z) * v - rv * s->g[2];
        }
        if (D->bc_top == 0 && i_z >= wall0_iz) f_p.z = 0.0;
        s->force[i].x += f_p.x; s->force[i].y += f_p.y; s->force[i].z += f_p.z;
        s->force[i].w += 0.0;
        d4 fp = {f_p.x, f_p.y, f_p.z, 0.0};
        D->f_p[i] = fp;
    }
}

/* findDarcyPermeabilities, darcy.cuh:1266-1313 */
static void permeabilities(const orc_state *s, struct orc_darcy *D)
{
    (void)s;
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) {
                unsigned c = didx(D, x, y, z);
                double phi = D->phi[c];
                if (phi > 0.9999) phi = 0.9999;
                double k = D->k_c * ORC_CUBE(phi) / ORC_SQUARE(1.0 - phi);
                D->k[c] = fmin(2.7e-10, k);
            }
}

/* findDarcyPermeabilityGradients, darcy.cuh:1316-1374 */
static void permeability_gradients(const orc_state *s, struct orc_darcy *D)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double *g = &D->grad_k[3 * (size_t)didx(D, x, y, z)];
                g[0] = (D->k[didx(D, x + 1, y, z)] - D->k[didx(D, x - 1, y, z)]) / (dx + dx);
                g[1] = (D->k[didx(D, x, y + 1, z)] - D->k[didx(D, x, y - 1, z)]) / (dy + dy);
                g[2] = (D->k[didx(D, x, y, z + 1)] - D->k[didx(D, x, y, z - 1)]) / (dz + dz);
            }
}

/* the pressure change of firstDarcySolution / updateDarcySolution
 * (darcy.cuh:1425-1598, 1602-1799) from the pressure field `pf` */
static double dp_of(const orc_state *s, const struct orc_darcy *D, const double *pf, int x, int y,
                    int z)
{
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    unsigned c = didx(D, x, y, z);
    double phi_xn = D->phi[didx(D, x - 1, y, z)], phi = D->phi[c];
    double phi_xp = D->phi[didx(D, x + 1, y, z)], phi_yn = D->phi[didx(D, x, y - 1, z)];
    double phi_yp = D->phi[didx(D, x, y + 1, z)], phi_zn = D->phi[didx(D, x, y, z - 1)];
    double phi_zp = D->phi[didx(D, x, y, z + 1)];
    double dphi = D->dphi[c];
    const double *vp = &D->vp_avg[3 * (size_t)c];
    int p_constant = D->p_constant[c];
    double p_xn = pf[didx(D, x - 1, y, z)], p = pf[c], p_xp = pf[didx(D, x + 1, y, z)];
    double p_yn = pf[didx(D, x, y - 1, z)], p_yp = pf[didx(D, x, y + 1, z)];
    double p_zn = pf[didx(D, x, y, z - 1)], p_zp = pf[didx(D, x, y, z + 1)];
    double k_xn = D->k[didx(D, x - 1, y, z)], k = D->k[c], k_xp = D->k[didx(D, x + 1, y, z)];
    double k_yn = D->k[didx(D, x, y - 1, z)], k_yp = D->k[didx(D, x, y + 1, z)];
    double k_zn = D->k[didx(D, x, y, z - 1)], k_zp = D->k[didx(D, x, y, z + 1)];
    if (x == 0 && D->bc_xn == 1) p_xn = p;
    if (x == nx - 1 && D->bc_xp == 1) p_xp = p;
    if (y == 0 && D->bc_yn == 1) p_yn = p;
    if (y == ny - 1 && D->bc_yp == 1) p_yp = p;
    if (z == 0 && D->bc_bot == 1) p_zn = p;
    if (z == nz - 1 && D->bc_top == 1) p_zp = p;
    double gx = (phi_xp - phi_xn) / (dx + dx), gy = (phi_yp - phi_yn) / (dy + dy),
           gz = (phi_zp - phi_zn) / (dz + dz);
    double div_k_grad_p =
        (2. * k_xp * k / (k_xp + k) * (p_xp - p) / dx - 2. * k_xn * k / (k_xn + k) * (p - p_xn) / dx) / dx +
        (2. * k_yp * k / (k_yp + k) * (p_yp - p) / dy - 2. * k_yn * k / (k_yn + k) * (p - p_yn) / dy) / dy +
        (2. * k_zp * k / (k_zp + k) * (p_zp - p) / dz - 2. * k_zn * k / (k_zn + k) * (p - p_zn) / dz) / dz;
    double ndt = D->ndem * s->dt;
    double dp = ndt / (D->beta_f * phi * D->mu) * div_k_grad_p -
                (ndt / (D->beta_f * phi * (1.0 - phi))) *
                    (dphi / ndt + (vp[0] * gx + vp[1] * gy + vp[2] * gz));
    if ((D->bc_bot == 0 && z == 0) || (D->bc_top == 0 && z == nz - 1) ||
        ((unsigned)z >= D->wall0_iz && D->bc_top == 0) || (D->bc_xn == 0 && x == 0) ||
        (D->bc_xp == 0 && x == nx - 1) || (D->bc_yn == 0 && y == 0) ||
        (D->bc_yp == 0 && y == nx - 1) || p_constant == 1)
        dp = 0.0;
    return dp;
}

/* maxNormResDarcy, darcy.cpp:266-292 (a maximum: the order of the scan
 * does not change it) */
static double max_norm(orc_state *s, struct orc_darcy *D, int *nan)
{
    double m = -1.0e9;
    int bad = 0;
#pragma omp parallel for reduction(max : m) reduction(| : bad) schedule(static)
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x) {
                double v = fabs(D->norm[didx(D, x, y, z)]);
                if (v != v) bad = 1;
                else if (v > m) m = v;
            }
    (void)s;
    *nan = bad;
    return m;
}

/* the Darcy block of the time loop, device.cu:1901-2426 */
int orc_darcy_step(orc_state *s)
{
    struct orc_darcy *D = s->darcy;
    const int nx = D->nx, ny = D->ny, nz = D->nz;
    if (s->nw > 0 && (s->wmode[0] == 1 || s->wmode[0] == 3))
        D->wall0_iz = (unsigned)(s->host_wall0_w / (s->L[2] / s->num[2]));
    if (s->np > 0) {
        ghost(s, D, D->p, 1);
        pressure_gradient(s, D);
        ghost(s, D, D->grad_p, 3);
        pressure_force(s, D);
    }
    if ((s->iter % D->ndem) != 0) return 0;
    porosities(s, D);
    if (s->periodic == 2) copy_edges(s, D);
    if ((D->p_mod_A > 1.0e-5 || D->p_mod_A < -1.0e-5) && D->p_mod_f > 1.0e-7) {
        double np_ = D->p_top_orig + D->p_mod_A * sin(2.0 * M_PI * D->p_mod_f * s->t_current + D->p_mod_phi);
        /* setDarcyTopPressure / setDarcyTopWallPressure (darcy.cuh:1195-1240),
         * restricted to cells inside the grid */
        for (int z = 0; z < nz + 8; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                    if (z == nz - 1 || (unsigned)z == D->wall0_iz)
                        if ((unsigned)z <= (unsigned)nz) D->p[didx(D, x, y, z)] = np_;
    }
    permeabilities(s, D);
    ghost(s, D, D->phi, 1);
    ghost(s, D, D->k, 1);
    permeability_gradients(s, D);
    if (s->iter == 0) {
        for (size_t i = 0; i < D->ng; ++i) D->norm[i] = 0.0;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) D->p_old[didx(D, x, y, z)] = D->p[didx(D, x, y, z)];
    }
    int flux = D->bc_bot == 4 || D->bc_top == 4;
    if (flux) ghost_flux(s, D);
    int64_t done = 0;
    for (unsigned nijac = 0; nijac < D->maxiter; ++nijac) {
        if (nijac == 0)
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x) D->p_old[didx(D, x, y, z)] = D->p[didx(D, x, y, z)];
        ghost(s, D, D->p, 1);
        if (nijac == 0)
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x) D->dp_expl[didx(D, x, y, z)] = dp_of(s, D, D->p, x, y, z);
        /* every cell reads the previous iterate only: the cells are independent */
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    unsigned c = didx(D, x, y, z);
                    double dp_impl = dp_of(s, D, D->p, x, y, z);
                    const double epsilon = 0.5, theta = 0.05;
                    double p = D->p[c];
                    double p_new = D->p_old[c] + (1.0 - epsilon) * D->dp_expl[c] + epsilon * dp_impl;
                    p_new = p * (1.0 - theta) + p_new * theta;
                    D->p_new[c] = p_new;
                    D->norm[c] = (p_new - p) / (p + 1.0e-16);
                }
        if (D->bc_top == 1) {
            /* setDarcyTopWallFixedFlow, darcy.cuh:1243-1262 */
            unsigned zz = D->wall0_iz + 1u;
            if (zz <= (unsigned)nz && zz >= 1u)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x)
                        D->p[didx(D, x, y, (int)zz)] = D->p[didx(D, x, y, (int)zz - 2)];
        }
        if (flux) ghost_flux(s, D);
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) D->p[didx(D, x, y, z)] = D->p_new[didx(D, x, y, z)];
        done = nijac;
        if (D->exact_stop || nijac % 10 == 0) {
            int nan;
            double m = max_norm(s, D, &nan);
            if (nan) {
                orc_set_error(s, ORC_ERR_INPUT, "Darcy residual is NaN");
                return s->err;
            }
            if (m <= D->tolerance) break;
        }
    }
    D->nijac_last = done;
    D->nijac_total += done + 1;
    if (s->filetimeclock + s->dt < s->file_dt)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) D->dphi[didx(D, x, y, z)] = 0.0;
    ghost(s, D, D->p, 1);
    /* findDarcyVelocities, darcy.cuh:1839-1897 */
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                unsigned c = didx(D, x, y, z);
                double gx = (D->p[didx(D, x + 1, y, z)] - D->p[didx(D, x - 1, y, z)]) / (dx + dx);
                double gy = (D->p[didx(D, x, y + 1, z)] - D->p[didx(D, x, y - 1, z)]) / (dy + dy);
                double gz = (D->p[didx(D, x, y, z + 1)] - D->p[didx(D, x, y, z - 1)]) / (dz + dz);
                double a = -D->k[c] / D->mu;
                D->v[3 * (size_t)c] = (a * gx) / D->phi[c];
                D->v[3 * (size_t)c + 1] = (a * gy) / D->phi[c];
                D->v[3 * (size_t)c + 2] = (a * gz) / D->phi[c];
            }
    return 0;
}

int64_t orc_darcy_get(orc_state *s, const char *name, void *dst, size_t bytes)
{
    struct orc_darcy *D = s->darcy;
    if (!D) return -1;
    size_t nc = (size_t)D->nx * D->ny * D->nz;
    if (!strcmp(name, "darcy_nijac_last") || !strcmp(name, "darcy_nijac_total")) {
        if (!dst || bytes < 8) return 8;
        int64_t v = !strcmp(name, "darcy_nijac_last") ? D->nijac_last : D->nijac_total;
        memcpy(dst, &v, 8);
        return 0;
    }
    if (!strcmp(name, "darcy_f_p")) {
        size_t need = (size_t)s->np * 32;
        if (!dst || bytes < need) return (int64_t)need;
        memcpy(dst, D->f_p, need);
        return 0;
    }
    const double *f = NULL;
    int comps = 1;
    if (!strcmp(name, "darcy_p")) f = D->p;
    else if (!strcmp(name, "darcy_phi")) f = D->phi;
    else if (!strcmp(name, "darcy_dphi")) f = D->dphi;
    else if (!strcmp(name, "darcy_k")) f = D->k;
    else if (!strcmp(name, "darcy_norm")) f = D->norm;
    else if (!strcmp(name, "darcy_v")) { f = D->v; comps = 3; }
    else if (!strcmp(name, "darcy_vp_avg")) { f = D->vp_avg; comps = 3; }
    else return -1;
    size_t need = nc * comps * 8;
    if (!dst || bytes < need) return (int64_t)need;
    double *o = (double *)dst;
    for (int z = 0; z < D->nz; ++z)
        for (int y = 0; y < D->ny; ++y)
            for (int x = 0; x < D->nx; ++x)
                for (int c = 0; c < comps; ++c)
                    o[(((size_t)z * D->ny + y) * D->nx + x) * comps + c] = f[(size_t)didx(D, x, y, z) * comps + c];
    return 0;
}

/* Option flags of the Darcy block: "darcy_exact_stop" (one int). */
int orc_darcy_set(orc_state *s, const char *name, const void *src, size_t bytes)
{
    struct orc_darcy *D = s->darcy;
    if (!D) return -1;
    if (!strcmp(name, "darcy_exact_stop") && bytes == sizeof(int)) {
        memcpy(&D->exact_stop, src, sizeof(int));
        return 0;
    }
    return -1;
}
