/* Internal state of the CPU oracle -- TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_INTERNAL_H_
#define ORACLE_INTERNAL_H_

#include <stdint.h>
#include <stddef.h>

/* The reference's PI constant (src/constants.h:15), not M_PI. */
#define ORC_PI 3.14159265358979

typedef struct { double x, y, z, w; } d4;
typedef struct { double x, y, z; } v3;

struct orc_state {
    /* header and grid (datatypes.h:45-63) */
    unsigned np, nd;
    double dt, t_current, t_total, file_dt;
    unsigned step_count;
    double origo[3], L[3];
    unsigned num[3];
    int periodic, adaptive;
    unsigned ncells;

    /* particle state, original order, the reference's Float4 layout */
    d4 *x, *xyzsum, *vel, *force, *angpos, *angvel, *torque, *acc, *angacc;
    double *es_dot, *es, *ev_dot, *ev, *p;
    int *color;

    /* parameters (datatypes.h:74-101) */
    double g[3], k_n, k_t, k_r, E, gamma_n, gamma_t, gamma_r, mu_s, mu_d,
        mu_r, gamma_wn, gamma_wt, mu_ws, mu_wd, rho;
    unsigned contactmodel;
    double kappa, db, V_b;

    /* walls (datatypes.h:104-110) */
    unsigned nw;
    int wmode[6];
    d4 wnx[6], wmvfd[6];
    double w_acc[6];
    double sigma0_A, sigma0_f, tau_x;

    /* bonds */
    double lambda_bar, sigma_b, tau_b;
    unsigned nb0;
    unsigned *bonds;   /* nb0 * 2 */
    d4 *bonds_delta;   /* (t.x, t.y, t.z, n) */
    d4 *bonds_omega;

    /* work arrays */
    unsigned *cellid, *index, *cellstart, *cellend;
    unsigned *sort_count, *sort_key, *sort_val;
    d4 *x_sorted, *vel_sorted, *angvel_sorted;
    unsigned nc;            /* contact slots per particle */
    unsigned *contacts;     /* np * nc, keyed by original index */
    d4 *distmod, *delta_t;  /* np * nc */
    double *walls_force_pp; /* nw * np */
    double *tau_eff_pp;     /* np */
    unsigned nblocks;       /* ceil(np / 256) */
    double *force_partials, *tau_partials;
    int capacity_hit;

    /* loop state */
    int64_t iter;
    int velocity_state;
    double filetimeclock;   /* time since the last file output */
    double host_wall0_w;    /* wall-0 position as of the last file output */

    /* options */
    int precision, integrator;

    /* fluid (Darcy, cfd_solver == 1) */
    int fluid, cfd_solver;
    struct orc_darcy *darcy;

    int err;
    char errmsg[256];
};

double orc_len(const struct orc_state *s, v3 v);
double orc_sqrtf(const struct orc_state *s, double v);
void orc_set_error(struct orc_state *s, int code, const char *msg);
void orc_block_sums(const double *in, unsigned n, double *out, unsigned nblocks);
void orc_bonds(struct orc_state *s);
int orc_darcy_step(struct orc_state *s);
int orc_darcy_load(struct orc_state *s, const unsigned char **cur,
                   const unsigned char *end);
int orc_darcy_write(struct orc_state *s, void *fh);
void orc_darcy_free(struct orc_state *s);
int64_t orc_darcy_get(struct orc_state *s, const char *name, void *dst, size_t bytes);
int orc_darcy_set(struct orc_state *s, const char *name, const void *src, size_t bytes);

#endif
