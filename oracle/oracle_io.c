/*
 * .bin loading, field access and writing for the CPU oracle -- TEST
 * INFRASTRUCTURE ONLY.  The byte layout follows src/file_io.cpp:30-417
 * (read) and :420-731 (write); this independent reader also cross-checks the
 * product's codec in the tests.
 */
#include "sph_oracle.h"
#include "oracle_internal.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const unsigned char *p, *end;
    int bad;
} rd;

static void take(rd *r, void *dst, size_t n)
{
    if (r->bad || (size_t)(r->end - r->p) < n) {
        r->bad = 1;
        memset(dst, 0, n);
        return;
    }
    memcpy(dst, r->p, n);
    r->p += n;
}
static double rf8(rd *r) { double v; take(r, &v, 8); return v; }
static unsigned ru4(rd *r) { unsigned v; take(r, &v, 4); return v; }
static int ri4(rd *r) { int v; take(r, &v, 4); return v; }

static void *xcalloc(size_t n, size_t sz)
{
    void *p = calloc(n ? n : 1, sz);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

void orc_free(orc_state *s)
{
    if (!s) return;
    free(s->x); free(s->xyzsum); free(s->vel); free(s->force); free(s->angpos);
    free(s->angvel); free(s->torque); free(s->acc); free(s->angacc);
    free(s->es_dot); free(s->es); free(s->ev_dot); free(s->ev); free(s->p);
    free(s->color); free(s->bonds); free(s->bonds_delta); free(s->bonds_omega);
    free(s->cellid); free(s->index); free(s->cellstart); free(s->cellend);
    free(s->sort_count); free(s->sort_key); free(s->sort_val);
    free(s->x_sorted); free(s->vel_sorted); free(s->angvel_sorted);
    free(s->contacts); free(s->distmod); free(s->delta_t);
    free(s->walls_force_pp); free(s->tau_eff_pp);
    free(s->force_partials); free(s->tau_partials);
    orc_darcy_free(s);
    free(s);
}

orc_state *orc_load(const char *path, int fluid, int precision, int integrator,
                    int nc, int *status)
{
    *status = ORC_OK;
    FILE *fh = fopen(path, "rb");
    if (!fh) { *status = ORC_ERR_FILE; return NULL; }
    fseek(fh, 0, SEEK_END);
    long len = ftell(fh);
    fseek(fh, 0, SEEK_SET);
    unsigned char *buf = (unsigned char *)xcalloc((size_t)len, 1);
    if (fread(buf, 1, (size_t)len, fh) != (size_t)len) {
        fclose(fh); free(buf); *status = ORC_ERR_FILE; return NULL;
    }
    fclose(fh);
    rd r = {buf, buf + len, 0};
    orc_state *s = (orc_state *)xcalloc(1, sizeof(orc_state));
    s->precision = precision;
    s->integrator = integrator == 2 ? 2 : 3;
    s->nc = nc > 0 ? (unsigned)nc : 32;
    s->velocity_state = 1;

    double version = rf8(&r);
    if (version != 2.15) {
        free(buf); free(s); *status = ORC_ERR_VERSION; return NULL;
    }
    s->nd = ru4(&r);
    s->np = ru4(&r);
    s->dt = rf8(&r); s->t_current = rf8(&r); s->t_total = rf8(&r);
    s->file_dt = rf8(&r); s->step_count = ru4(&r);
    take(&r, s->origo, 24); take(&r, s->L, 24); take(&r, s->num, 12);
    s->periodic = ri4(&r); s->adaptive = ri4(&r);
    unsigned n = s->np;
    if (r.bad || s->nd != 3 || (uint64_t)n * 32 > (uint64_t)len) {
        free(buf); free(s); *status = ORC_ERR_INPUT; return NULL;
    }
    s->ncells = s->num[0] * s->num[1] * s->num[2];
    s->x = xcalloc(n, sizeof(d4)); s->xyzsum = xcalloc(n, sizeof(d4));
    s->vel = xcalloc(n, sizeof(d4)); s->force = xcalloc(n, sizeof(d4));
    s->angpos = xcalloc(n, sizeof(d4)); s->angvel = xcalloc(n, sizeof(d4));
    s->torque = xcalloc(n, sizeof(d4)); s->acc = xcalloc(n, sizeof(d4));
    s->angacc = xcalloc(n, sizeof(d4));
    s->es_dot = xcalloc(n, 8); s->es = xcalloc(n, 8); s->ev_dot = xcalloc(n, 8);
    s->ev = xcalloc(n, 8); s->p = xcalloc(n, 8); s->color = xcalloc(n, 4);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->x[i], 32);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->xyzsum[i], 24);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->vel[i], 32);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->force[i], 24);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->angpos[i], 24);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->angvel[i], 24);
    for (unsigned i = 0; i < n; ++i) take(&r, &s->torque[i], 24);
    take(&r, s->es_dot, 8 * (size_t)n); take(&r, s->es, 8 * (size_t)n);
    take(&r, s->ev_dot, 8 * (size_t)n); take(&r, s->ev, 8 * (size_t)n);
    take(&r, s->p, 8 * (size_t)n);
    take(&r, s->g, 24);
    s->k_n = rf8(&r); s->k_t = rf8(&r); s->k_r = rf8(&r); s->E = rf8(&r);
    s->gamma_n = rf8(&r); s->gamma_t = rf8(&r); s->gamma_r = rf8(&r);
    s->mu_s = rf8(&r); s->mu_d = rf8(&r); s->mu_r = rf8(&r);
    s->gamma_wn = rf8(&r); s->gamma_wt = rf8(&r);
    s->mu_ws = rf8(&r); s->mu_wd = rf8(&r); s->rho = rf8(&r);
    s->contactmodel = ru4(&r);
    s->kappa = rf8(&r); s->db = rf8(&r); s->V_b = rf8(&r);
    s->nw = ru4(&r);
    if (s->nw > 6) { free(buf); orc_free(s); *status = ORC_ERR_INPUT; return NULL; }
    for (unsigned w = 0; w < s->nw; ++w) s->wmode[w] = ri4(&r);
    for (unsigned w = 0; w < s->nw; ++w) take(&r, &s->wnx[w], 32);
    for (unsigned w = 0; w < s->nw; ++w) take(&r, &s->wmvfd[w], 32);
    s->sigma0_A = rf8(&r); s->sigma0_f = rf8(&r); s->tau_x = rf8(&r);
    s->lambda_bar = rf8(&r); s->nb0 = ru4(&r); s->sigma_b = rf8(&r);
    s->tau_b = rf8(&r);
    unsigned nb = s->nb0;
    if ((uint64_t)nb * 8 > (uint64_t)len) { free(buf); orc_free(s); *status = ORC_ERR_INPUT; return NULL; }
    s->bonds = xcalloc((size_t)nb * 2, 4);
    s->bonds_delta = xcalloc(nb, sizeof(d4));
    s->bonds_omega = xcalloc(nb, sizeof(d4));
    take(&r, s->bonds, 8 * (size_t)nb);
    for (unsigned i = 0; i < nb; ++i) s->bonds_delta[i].w = rf8(&r);
    for (unsigned i = 0; i < nb; ++i) take(&r, &s->bonds_delta[i], 24);
    for (unsigned i = 0; i < nb; ++i) s->bonds_omega[i].w = rf8(&r);
    for (unsigned i = 0; i < nb; ++i) take(&r, &s->bonds_omega[i], 24);
    s->fluid = fluid;
    if (fluid) {
        s->cfd_solver = ri4(&r);
        if (s->cfd_solver != 1) {
            free(buf); orc_free(s); *status = ORC_ERR_UNSUPPORTED; return NULL;
        }
        const unsigned char *cur = r.p;
        int rc = orc_darcy_load(s, &cur, r.end);
        if (rc) { free(buf); orc_free(s); *status = rc; return NULL; }
        r.p = cur;
    }
    take(&r, s->color, 4 * (size_t)n);
    if (r.bad || r.p != r.end) {
        free(buf); orc_free(s); *status = ORC_ERR_INPUT; return NULL;
    }
    free(buf);

    /* work arrays (device.cu:405-487; history zero-initialised) */
    s->cellid = xcalloc(n, 4); s->index = xcalloc(n, 4);
    s->cellstart = xcalloc(s->ncells, 4); s->cellend = xcalloc(s->ncells, 4);
    s->sort_count = xcalloc((size_t)s->ncells + 1, 4);
    s->sort_key = xcalloc(n, 4); s->sort_val = xcalloc(n, 4);
    s->x_sorted = xcalloc(n, sizeof(d4)); s->vel_sorted = xcalloc(n, sizeof(d4));
    s->angvel_sorted = xcalloc(n, sizeof(d4));
    size_t nslots = (size_t)n * s->nc;
    s->contacts = xcalloc(nslots, 4);
    for (size_t i = 0; i < nslots; ++i) s->contacts[i] = n;
    s->distmod = xcalloc(nslots, sizeof(d4));
    s->delta_t = xcalloc(nslots, sizeof(d4));
    s->walls_force_pp = xcalloc((size_t)n * (s->nw ? s->nw : 1), 8);
    s->tau_eff_pp = xcalloc(n, 8);
    s->nblocks = (n + 255) / 256;
    s->force_partials = xcalloc(s->nblocks, 8);
    s->tau_partials = xcalloc(s->nblocks, 8);
    for (unsigned i = 0; i < n; ++i) {
        s->force[i].w = 0; s->angpos[i].w = 0; s->angvel[i].w = 0;
        s->torque[i].w = 0; s->xyzsum[i].w = 0;
    }
    return s;
}

#define FIELD4(nm, arr, cnt)                                                  \
    if (!strcmp(name, nm)) { ptr = (void *)(arr); need = (size_t)(cnt) * 32; }
#define FIELDN(nm, arr, cnt, sz)                                              \
    if (!strcmp(name, nm)) { ptr = (void *)(arr); need = (size_t)(cnt) * (sz); }

static int64_t locate(orc_state *s, const char *name, void **pptr)
{
    void *ptr = NULL;
    size_t need = 0;
    unsigned n = s->np;
    size_t slots = (size_t)n * s->nc;
    FIELD4("x", s->x, n) FIELD4("vel", s->vel, n) FIELD4("angvel", s->angvel, n)
    FIELD4("angpos", s->angpos, n) FIELD4("force", s->force, n)
    FIELD4("torque", s->torque, n) FIELD4("acc", s->acc, n)
    FIELD4("angacc", s->angacc, n) FIELD4("xyzsum", s->xyzsum, n)
    FIELDN("es_dot", s->es_dot, n, 8) FIELDN("es", s->es, n, 8)
    FIELDN("ev_dot", s->ev_dot, n, 8) FIELDN("ev", s->ev, n, 8)
    FIELDN("p", s->p, n, 8)
    FIELDN("cellid", s->cellid, n, 4) FIELDN("index", s->index, n, 4)
    FIELDN("cellstart", s->cellstart, s->ncells, 4)
    FIELDN("cellend", s->cellend, s->ncells, 4)
    FIELDN("contacts", s->contacts, slots, 4)
    FIELD4("delta_t", s->delta_t, slots) FIELD4("distmod", s->distmod, slots)
    FIELD4("walls_nx", s->wnx, s->nw) FIELD4("walls_mvfd", s->wmvfd, s->nw)
    FIELDN("walls_acc", s->w_acc, s->nw, 8)
    FIELDN("walls_force_partial", s->force_partials, s->nblocks, 8)
    FIELDN("iter", &s->iter, 1, 8) FIELDN("time", &s->t_current, 1, 8)
    FIELDN("bonds", s->bonds, (size_t)s->nb0 * 2, 4)
    FIELD4("bonds_delta", s->bonds_delta, s->nb0)
    FIELD4("bonds_omega", s->bonds_omega, s->nb0)
    if (!ptr) return -1;
    *pptr = ptr;
    return (int64_t)need;
}

int64_t orc_get(orc_state *s, const char *name, void *dst, size_t bytes)
{
    if (!strncmp(name, "darcy_", 6)) return orc_darcy_get(s, name, dst, bytes);
    void *ptr;
    int64_t need = locate(s, name, &ptr);
    if (need < 0) return -1;
    if (!dst || bytes < (size_t)need) return need ? need : 0;
    memcpy(dst, ptr, (size_t)need);
    return 0;
}

int orc_set(orc_state *s, const char *name, const void *src, size_t bytes)
{
    if (!strncmp(name, "darcy_exact_stop", 16)) return orc_darcy_set(s, name, src, bytes);
    void *ptr;
    int64_t need = locate(s, name, &ptr);
    if (need < 0 || bytes != (size_t)need) return -1;
    memcpy(ptr, src, bytes);
    return 0;
}

static void wf8(FILE *f, double v) { fwrite(&v, 8, 1, f); }
static void wu4(FILE *f, unsigned v) { fwrite(&v, 4, 1, f); }
static void wi4(FILE *f, int v) { fwrite(&v, 4, 1, f); }

/* writebin, src/file_io.cpp:420-731 */
int orc_write_bin(orc_state *s, const char *path)
{
    FILE *f = fopen(path, "wb");
    if (!f) return ORC_ERR_FILE;
    unsigned n = s->np;
    wf8(f, 2.15); wu4(f, s->nd); wu4(f, n);
    wf8(f, s->dt); wf8(f, s->t_current); wf8(f, s->t_total); wf8(f, s->file_dt);
    wu4(f, s->step_count);
    fwrite(s->origo, 8, 3, f); fwrite(s->L, 8, 3, f); fwrite(s->num, 4, 3, f);
    wi4(f, s->periodic); wi4(f, s->adaptive);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->x[i], 8, 4, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->xyzsum[i], 8, 3, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->vel[i], 8, 4, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->force[i], 8, 3, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->angpos[i], 8, 3, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->angvel[i], 8, 3, f);
    for (unsigned i = 0; i < n; ++i) fwrite(&s->torque[i], 8, 3, f);
    fwrite(s->es_dot, 8, n, f); fwrite(s->es, 8, n, f); fwrite(s->ev_dot, 8, n, f);
    fwrite(s->ev, 8, n, f); fwrite(s->p, 8, n, f);
    fwrite(s->g, 8, 3, f);
    double pr[] = {s->k_n, s->k_t, s->k_r, s->E, s->gamma_n, s->gamma_t,
                   s->gamma_r, s->mu_s, s->mu_d, s->mu_r, s->gamma_wn,
                   s->gamma_wt, s->mu_ws, s->mu_wd, s->rho};
    fwrite(pr, 8, 15, f);
    wu4(f, s->contactmodel);
    wf8(f, s->kappa); wf8(f, s->db); wf8(f, s->V_b);
    wu4(f, s->nw);
    for (unsigned w = 0; w < s->nw; ++w) wi4(f, s->wmode[w]);
    for (unsigned w = 0; w < s->nw; ++w) fwrite(&s->wnx[w], 8, 4, f);
    for (unsigned w = 0; w < s->nw; ++w) fwrite(&s->wmvfd[w], 8, 4, f);
    wf8(f, s->sigma0_A); wf8(f, s->sigma0_f); wf8(f, s->tau_x);
    wf8(f, s->lambda_bar); wu4(f, s->nb0); wf8(f, s->sigma_b); wf8(f, s->tau_b);
    fwrite(s->bonds, 4, (size_t)s->nb0 * 2, f);
    for (unsigned i = 0; i < s->nb0; ++i) wf8(f, s->bonds_delta[i].w);
    for (unsigned i = 0; i < s->nb0; ++i) fwrite(&s->bonds_delta[i], 8, 3, f);
    for (unsigned i = 0; i < s->nb0; ++i) wf8(f, s->bonds_omega[i].w);
    for (unsigned i = 0; i < s->nb0; ++i) fwrite(&s->bonds_omega[i], 8, 3, f);
    if (s->fluid) {
        wi4(f, s->cfd_solver);
        orc_darcy_write(s, f);
    }
    fwrite(s->color, 4, n, f);
    fclose(f);
    /* a file output refreshes the host copy of the wall and the clock */
    if (s->nw > 0) s->host_wall0_w = s->wnx[0].w;
    s->filetimeclock = 0.0;
    return 0;
}
