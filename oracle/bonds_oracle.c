/*
 * Parallel-bond forces for the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 * Restates bondsLinear (src/cohesion.cuh:8-233).  The reference accumulates
 * bond forces with unsynchronised `+=` from one thread per bond
 * (cohesion.cuh:220-226); the oracle defines the result as the serial
 * accumulation in bond order.
 */
#include "sph_oracle.h"
#include "oracle_internal.h"

#include <math.h>

static inline v3 mk3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
static inline v3 smul3(double b, v3 a) { return mk3(b * a.x, b * a.y, b * a.z); }
static inline v3 muls3(v3 a, double b) { return mk3(a.x * b, a.y * b, a.z * b); }
static inline v3 divs3(v3 a, double b) { return mk3(a.x / b, a.y / b, a.z / b); }
static inline double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

void orc_bonds(orc_state *s)
{
    const double dt = s->dt;
    for (unsigned idx = 0; idx < s->nb0; ++idx) {
        unsigned bx = s->bonds[2 * idx], by = s->bonds[2 * idx + 1];
        if (!(bx < s->np)) continue;
        if (by >= s->np) {
            orc_set_error(s, ORC_ERR_INPUT, "bond refers to a particle index >= np");
            return;
        }
        d4 d0 = s->bonds_delta[idx], w0 = s->bonds_omega[idx];
        v3 delta0_t = mk3(d0.x, d0.y, d0.z);
        double delta0_n = d0.w;
        v3 omega0_t = mk3(w0.x, w0.y, w0.z);
        double omega0_n = w0.w;
        d4 x_i = s->x[bx], x_j = s->x[by];
        d4 vel_i = s->vel[bx], vel_j = s->vel[by];
        v3 angvel_i = mk3(s->angvel[bx].x, s->angvel[bx].y, s->angvel[bx].z);
        v3 angvel_j = mk3(s->angvel[by].x, s->angvel[by].y, s->angvel[by].z);

        double R_bar = s->lambda_bar * fmin(x_i.w, x_j.w);
        double A = ORC_PI * R_bar * R_bar;
        double I = 0.25 * ORC_PI * R_bar * R_bar * R_bar * R_bar;
        double J = I * 2.0;
        v3 x = mk3(x_i.x - x_j.x, x_i.y - x_j.y, x_i.z - x_j.z);
        double x_length = orc_len(s, x);
        double overlap = fmin(0.0, x_length - (x_i.w + x_j.w));
        v3 n = divs3(x, x_length);
        delta0_t = sub3(delta0_t, muls3(n, dot3(n, delta0_t)));
        v3 ddelta = muls3(add3(add3(mk3(vel_i.x - vel_j.x, vel_i.y - vel_j.y,
                                        vel_i.z - vel_j.z),
                                    smul3(x_i.w + overlap / 2.0, cross3(n, angvel_i))),
                               smul3(x_j.w + overlap / 2.0, cross3(n, angvel_j))),
                          dt);
        double ddelta_n = -dot3(ddelta, n);
        double delta_n = delta0_n + ddelta_n;
        v3 ddelta_t = sub3(ddelta, muls3(n, dot3(n, ddelta)));
        v3 delta_t = add3(delta0_t, ddelta_t);
        v3 f_n = smul3(s->k_n * A * delta_n + s->gamma_n * ddelta_n / dt, n);
        v3 f_t = sub3(smul3(-s->k_t * A, delta_t), divs3(smul3(s->gamma_t, ddelta_t), dt));
        v3 f = add3(f_n, f_t);
        v3 nn = neg3(n);
        omega0_t = sub3(omega0_t, muls3(nn, dot3(omega0_t, nn)));
        v3 domega = muls3(mk3(angvel_j.x - angvel_i.x, angvel_j.y - angvel_i.y,
                              angvel_j.z - angvel_i.z), dt);
        double domega_n = dot3(domega, nn);
        double omega_n = omega0_n + domega_n;
        v3 domega_t = sub3(domega, smul3(domega_n, nn));
        v3 omega_t = add3(omega0_t, domega_t);
        v3 t_n = smul3(-s->k_t * J * omega_n, nn);
        v3 t_t = smul3(-s->k_n * I, omega_t);
        v3 t_j = add3(t_n, t_t);
        double sigma_max = orc_len(s, f_n) / A + orc_len(s, t_t) * R_bar / I;
        double tau_max = orc_len(s, f_t) / A + orc_len(s, t_n) * R_bar / J;
        if (sigma_max >= s->sigma_b || tau_max >= s->tau_b) {
            /* the reference marks a broken bond with nb0 (cohesion.cuh:205) */
            s->bonds[2 * idx] = s->nb0;
            continue;
        }
        d4 nd = {delta_t.x, delta_t.y, delta_t.z, delta_n};
        d4 nw = {omega_t.x, omega_t.y, omega_t.z, omega_n};
        s->bonds_delta[idx] = nd;
        s->bonds_omega[idx] = nw;
        s->force[bx].x += f.x; s->force[bx].y += f.y; s->force[bx].z += f.z;
        s->force[bx].w += 0.0;
        s->force[by].x -= f.x; s->force[by].y -= f.y; s->force[by].z -= f.z;
        s->force[by].w -= 0.0;
        s->torque[bx].x -= t_j.x; s->torque[bx].y -= t_j.y; s->torque[bx].z -= t_j.z;
        s->torque[bx].w -= 0.0;
        s->torque[by].x += t_j.x; s->torque[by].y += t_j.y; s->torque[by].z += t_j.z;
        s->torque[by].w += 0.0;
    }
}
