// Host-side copy of one sphere simulation (.bin contents), in the
// reference's layout: Float4 = 4 doubles per particle, original order.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace sphb {

struct d4 {
    double x, y, z, w;
};

struct HostState {
    // header, grid (src/datatypes.h:45-73)
    uint32_t nd = 3, np = 0;
    double dt = 0, t_current = 0, t_total = 0, file_dt = 0;
    uint32_t step_count = 0;
    double origo[3] = {0, 0, 0}, L[3] = {0, 0, 0};
    uint32_t num[3] = {0, 0, 0};
    int32_t periodic = 0, adaptive = 0;

    // particles
    std::vector<d4> x, xyzsum, vel, force, angpos, angvel, torque;
    std::vector<double> es_dot, es, ev_dot, ev, p;
    std::vector<int32_t> color;

    // parameters (src/datatypes.h:74-101)
    double g[3] = {0, 0, 0};
    double k_n = 0, k_t = 0, k_r = 0, E = 0, gamma_n = 0, gamma_t = 0,
           gamma_r = 0, mu_s = 0, mu_d = 0, mu_r = 0, gamma_wn = 0,
           gamma_wt = 0, mu_ws = 0, mu_wd = 0, rho = 0;
    uint32_t contactmodel = 2;
    double kappa = 0, db = 0, V_b = 0;

    // walls (src/datatypes.h:104-110)
    uint32_t nw = 0;
    int32_t wmode[6] = {0, 0, 0, 0, 0, 0};
    d4 wnx[6] = {}, wmvfd[6] = {};
    double sigma0_A = 0, sigma0_f = 0, tau_x = 0;

    // bonds
    double lambda_bar = 1, sigma_b = 0, tau_b = 0;
    uint32_t nb0 = 0;
    std::vector<uint32_t> bonds;       // 2 per bond
    std::vector<d4> bonds_delta;       // (t.x, t.y, t.z, n)
    std::vector<d4> bonds_omega;

    // fluid (src/datatypes.h:158-190): Darcy (cfd_solver 1) and
    // Navier-Stokes (cfd_solver 0) share the grid fields and most settings
    int fluid = 0;
    int32_t cfd_solver = 1;
    double mu = 0;
    std::vector<double> v_f;     // ncells*3, x fastest (file order)
    std::vector<double> p_f, phi, dphi;  // ncells
    double rho_f = 0, p_mod_A = 0, p_mod_f = 0, p_mod_phi = 0;
    int32_t bc_xn = 2, bc_xp = 2, bc_yn = 2, bc_yp = 2, bc_bot = 0, bc_top = 0;
    int32_t free_slip_bot = 1, free_slip_top = 1;
    double bc_bot_flux = 0, bc_top_flux = 0;
    std::vector<int32_t> p_constant;    // ncells
    double tolerance = 1e-3;
    uint32_t maxiter = 10000, ndem = 1;
    double c_phi = 1;
    std::vector<d4> f_p;               // np (w unused)
    double beta_f = 4.5e-10, k_c = 4.6e-10;
    // Navier-Stokes only: smoothing, relaxation, pressure-projection weight,
    // velocity prefactor, time step factor, and the per-particle drag,
    // viscous and total interaction forces (f_p above holds the pressure
    // force)
    double ns_gamma = 0, ns_theta = 1, ns_beta = 0, c_v = 1, dt_dem_fac = 1;
    std::vector<d4> f_d, f_v, f_sum;

    uint64_t ncells() const { return (uint64_t)num[0] * num[1] * num[2]; }
};

// Status codes shared with the C ABI.
enum Status {
    ST_OK = 0,
    ST_FILE = -1,
    ST_VERSION = -2,
    ST_INPUT = -3,
    ST_CUDA = -4,
    ST_OUTSIDE = -5,
    ST_CAPACITY = -6,
    ST_UNSUPPORTED = -7,
    ST_ARG = -8,
    ST_TIMEOUT = -9,
};

// Parses a .bin image (src/file_io.cpp:30-417).  `fluid` is the reference's
// --fluid flag.  Returns a Status; `err` gets a message.
int parse_bin(const uint8_t *buf, size_t len, int fluid, HostState &s, std::string &err);
int read_bin_file(const char *path, int fluid, HostState &s, std::string &err);
// Serialises (src/file_io.cpp:420-731); always format 2.15.
std::vector<uint8_t> serialize_bin(const HostState &s);
int write_bin_file(const char *path, const HostState &s, std::string &err);
// Input checks of DEM::checkValues (src/sphere.cpp:145-345), returned as a
// status instead of exit(1).
int check_values(const HostState &s, std::string &err);

}  // namespace sphb
