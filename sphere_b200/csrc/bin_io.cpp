// .bin v2.15 codec and input validation for the engine.
// Layout: src/file_io.cpp:30-417 (read), :420-731 (write).
#include "host_state.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace sphb {

namespace {

struct Reader {
    const uint8_t *p, *end;
    bool bad = false;
    void take(void *dst, size_t n)
    {
        if (bad || (size_t)(end - p) < n) {
            bad = true;
            std::memset(dst, 0, n);
            return;
        }
        std::memcpy(dst, p, n);
        p += n;
    }
    double f8() { double v; take(&v, 8); return v; }
    uint32_t u4() { uint32_t v; take(&v, 4); return v; }
    int32_t i4() { int32_t v; take(&v, 4); return v; }
    size_t left() const { return bad ? 0 : (size_t)(end - p); }
};

struct Writer {
    std::vector<uint8_t> out;
    void put(const void *src, size_t n)
    {
        const uint8_t *b = (const uint8_t *)src;
        out.insert(out.end(), b, b + n);
    }
    void f8(double v) { put(&v, 8); }
    void u4(uint32_t v) { put(&v, 4); }
    void i4(int32_t v) { put(&v, 4); }
};

}  // namespace

int parse_bin(const uint8_t *buf, size_t len, int fluid, HostState &s, std::string &err)
{
    Reader r{buf, buf + len};
    double version = r.f8();
    if (r.bad) { err = "file shorter than its header"; return ST_FILE; }
    if (version != 2.15) {
        char m[160];
        std::snprintf(m, sizeof m, "file written by sphere version %g, this engine reads 2.15", version);
        err = m;
        return ST_VERSION;
    }
    s.nd = r.u4();
    s.np = r.u4();
    s.dt = r.f8(); s.t_current = r.f8(); s.t_total = r.f8(); s.file_dt = r.f8();
    s.step_count = r.u4();
    r.take(s.origo, 24); r.take(s.L, 24); r.take(s.num, 12);
    s.periodic = r.i4(); s.adaptive = r.i4();
    if (r.bad) { err = "file truncated in header"; return ST_FILE; }
    if (s.nd != 3) { err = "dimensionality is not 3"; return ST_INPUT; }
    uint32_t n = s.np;
    // every particle needs at least 228 bytes; reject counts the file can't hold
    if ((uint64_t)n * 228 > len) { err = "particle count exceeds the file size"; return ST_FILE; }
    s.x.assign(n, d4{}); s.xyzsum.assign(n, d4{}); s.vel.assign(n, d4{});
    s.force.assign(n, d4{}); s.angpos.assign(n, d4{}); s.angvel.assign(n, d4{});
    s.torque.assign(n, d4{});
    for (uint32_t i = 0; i < n; ++i) r.take(&s.x[i], 32);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.xyzsum[i], 24);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.vel[i], 32);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.force[i], 24);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.angpos[i], 24);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.angvel[i], 24);
    for (uint32_t i = 0; i < n; ++i) r.take(&s.torque[i], 24);
    auto vecd = [&](std::vector<double> &v) { v.assign(n, 0.0); r.take(v.data(), 8 * (size_t)n); };
    vecd(s.es_dot); vecd(s.es); vecd(s.ev_dot); vecd(s.ev); vecd(s.p);
    r.take(s.g, 24);
    s.k_n = r.f8(); s.k_t = r.f8(); s.k_r = r.f8(); s.E = r.f8();
    s.gamma_n = r.f8(); s.gamma_t = r.f8(); s.gamma_r = r.f8();
    s.mu_s = r.f8(); s.mu_d = r.f8(); s.mu_r = r.f8();
    s.gamma_wn = r.f8(); s.gamma_wt = r.f8(); s.mu_ws = r.f8(); s.mu_wd = r.f8();
    s.rho = r.f8();
    s.contactmodel = r.u4();
    s.kappa = r.f8(); s.db = r.f8(); s.V_b = r.f8();
    s.nw = r.u4();
    if (r.bad) { err = "file truncated in the particle block"; return ST_FILE; }
    if (s.nw > 6) { err = "more walls than MAXWALLS (6)"; return ST_INPUT; }
    for (uint32_t w = 0; w < s.nw; ++w) s.wmode[w] = r.i4();
    for (uint32_t w = 0; w < s.nw; ++w) r.take(&s.wnx[w], 32);
    for (uint32_t w = 0; w < s.nw; ++w) r.take(&s.wmvfd[w], 32);
    s.sigma0_A = r.f8(); s.sigma0_f = r.f8(); s.tau_x = r.f8();
    s.lambda_bar = r.f8(); s.nb0 = r.u4(); s.sigma_b = r.f8(); s.tau_b = r.f8();
    if (r.bad) { err = "file truncated in the wall block"; return ST_FILE; }
    uint32_t nb = s.nb0;
    if ((uint64_t)nb * 72 > r.left()) { err = "bond count exceeds the file size"; return ST_FILE; }
    s.bonds.assign(2 * (size_t)nb, 0);
    r.take(s.bonds.data(), 8 * (size_t)nb);
    s.bonds_delta.assign(nb, d4{}); s.bonds_omega.assign(nb, d4{});
    for (uint32_t i = 0; i < nb; ++i) s.bonds_delta[i].w = r.f8();
    for (uint32_t i = 0; i < nb; ++i) r.take(&s.bonds_delta[i], 24);
    for (uint32_t i = 0; i < nb; ++i) s.bonds_omega[i].w = r.f8();
    for (uint32_t i = 0; i < nb; ++i) r.take(&s.bonds_omega[i], 24);
    s.fluid = fluid ? 1 : 0;
    if (fluid) {
        s.cfd_solver = r.i4();
        if (s.cfd_solver != 0 && s.cfd_solver != 1) {
            err = "cfd_solver value not understood";
            return ST_INPUT;
        }
        s.mu = r.f8();
        uint64_t nc = s.ncells();
        if (nc * 52 > r.left()) { err = "fluid grid exceeds the file size"; return ST_FILE; }
        s.v_f.assign(3 * nc, 0.0); s.p_f.assign(nc, 0.0);
        s.phi.assign(nc, 0.0); s.dphi.assign(nc, 0.0);
        for (uint64_t i = 0; i < nc; ++i) {
            r.take(&s.v_f[3 * i], 24);
            s.p_f[i] = r.f8(); s.phi[i] = r.f8(); s.dphi[i] = r.f8();
        }
        s.rho_f = r.f8(); s.p_mod_A = r.f8(); s.p_mod_f = r.f8(); s.p_mod_phi = r.f8();
        if (s.cfd_solver == 1) {
            s.bc_xn = r.i4(); s.bc_xp = r.i4(); s.bc_yn = r.i4(); s.bc_yp = r.i4();
            s.bc_bot = r.i4(); s.bc_top = r.i4();
        } else {
            // the Navier-Stokes block has no side conditions and names the
            // top condition first (src/file_io.cpp:297-298)
            s.bc_top = r.i4(); s.bc_bot = r.i4();
        }
        s.free_slip_bot = r.i4(); s.free_slip_top = r.i4();
        s.bc_bot_flux = r.f8(); s.bc_top_flux = r.f8();
        s.p_constant.assign(nc, 0);
        r.take(s.p_constant.data(), 4 * nc);
        if (s.cfd_solver == 0) {
            // src/file_io.cpp:306-336
            s.ns_gamma = r.f8(); s.ns_theta = r.f8(); s.ns_beta = r.f8();
            s.tolerance = r.f8(); s.maxiter = r.u4(); s.ndem = r.u4();
            s.c_phi = r.f8(); s.c_v = r.f8(); s.dt_dem_fac = r.f8();
            if ((uint64_t)n * 96 > r.left()) { err = "file truncated in the fluid forces"; return ST_FILE; }
            for (std::vector<d4> *a : {&s.f_d, &s.f_p, &s.f_v, &s.f_sum}) {
                a->assign(n, d4{});
                for (uint32_t i = 0; i < n; ++i) r.take(&(*a)[i], 24);
            }
        } else {
            s.tolerance = r.f8(); s.maxiter = r.u4(); s.ndem = r.u4(); s.c_phi = r.f8();
            s.f_p.assign(n, d4{});
            for (uint32_t i = 0; i < n; ++i) r.take(&s.f_p[i], 24);
            s.beta_f = r.f8(); s.k_c = r.f8();
        }
    }
    s.color.assign(n, 0);
    r.take(s.color.data(), 4 * (size_t)n);
    if (r.bad) { err = "file truncated"; return ST_FILE; }
    if (r.left() != 0) {
        err = "trailing bytes after the color block (fluid flag mismatch?)";
        return ST_FILE;
    }
    return ST_OK;
}

int read_bin_file(const char *path, int fluid, HostState &s, std::string &err)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) { err = std::string("could not read input binary file '") + path + "'"; return ST_FILE; }
    std::fseek(f, 0, SEEK_END);
    long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<uint8_t> buf(len > 0 ? (size_t)len : 0);
    size_t got = len > 0 ? std::fread(buf.data(), 1, (size_t)len, f) : 0;
    std::fclose(f);
    if ((long)got != len) { err = "short read"; return ST_FILE; }
    return parse_bin(buf.data(), buf.size(), fluid, s, err);
}

std::vector<uint8_t> serialize_bin(const HostState &s)
{
    Writer w;
    uint32_t n = s.np;
    w.f8(2.15); w.u4(s.nd); w.u4(n);
    w.f8(s.dt); w.f8(s.t_current); w.f8(s.t_total); w.f8(s.file_dt);
    w.u4(s.step_count);
    w.put(s.origo, 24); w.put(s.L, 24); w.put(s.num, 12);
    w.i4(s.periodic); w.i4(s.adaptive);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.x[i], 32);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.xyzsum[i], 24);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.vel[i], 32);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.force[i], 24);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.angpos[i], 24);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.angvel[i], 24);
    for (uint32_t i = 0; i < n; ++i) w.put(&s.torque[i], 24);
    w.put(s.es_dot.data(), 8 * (size_t)n); w.put(s.es.data(), 8 * (size_t)n);
    w.put(s.ev_dot.data(), 8 * (size_t)n); w.put(s.ev.data(), 8 * (size_t)n);
    w.put(s.p.data(), 8 * (size_t)n);
    w.put(s.g, 24);
    double pr[] = {s.k_n, s.k_t, s.k_r, s.E, s.gamma_n, s.gamma_t, s.gamma_r,
                   s.mu_s, s.mu_d, s.mu_r, s.gamma_wn, s.gamma_wt, s.mu_ws,
                   s.mu_wd, s.rho};
    w.put(pr, sizeof pr);
    w.u4(s.contactmodel);
    w.f8(s.kappa); w.f8(s.db); w.f8(s.V_b);
    w.u4(s.nw);
    for (uint32_t i = 0; i < s.nw; ++i) w.i4(s.wmode[i]);
    for (uint32_t i = 0; i < s.nw; ++i) w.put(&s.wnx[i], 32);
    for (uint32_t i = 0; i < s.nw; ++i) w.put(&s.wmvfd[i], 32);
    w.f8(s.sigma0_A); w.f8(s.sigma0_f); w.f8(s.tau_x);
    w.f8(s.lambda_bar); w.u4(s.nb0); w.f8(s.sigma_b); w.f8(s.tau_b);
    w.put(s.bonds.data(), 4 * s.bonds.size());
    for (uint32_t i = 0; i < s.nb0; ++i) w.f8(s.bonds_delta[i].w);
    for (uint32_t i = 0; i < s.nb0; ++i) w.put(&s.bonds_delta[i], 24);
    for (uint32_t i = 0; i < s.nb0; ++i) w.f8(s.bonds_omega[i].w);
    for (uint32_t i = 0; i < s.nb0; ++i) w.put(&s.bonds_omega[i], 24);
    if (s.fluid) {
        w.i4(s.cfd_solver);
        w.f8(s.mu);
        uint64_t nc = s.ncells();
        for (uint64_t i = 0; i < nc; ++i) {
            w.put(&s.v_f[3 * i], 24);
            w.f8(s.p_f[i]); w.f8(s.phi[i]); w.f8(s.dphi[i]);
        }
        w.f8(s.rho_f); w.f8(s.p_mod_A); w.f8(s.p_mod_f); w.f8(s.p_mod_phi);
        if (s.cfd_solver == 1) {
            w.i4(s.bc_xn); w.i4(s.bc_xp); w.i4(s.bc_yn); w.i4(s.bc_yp);
        }
        // bottom first, also for Navier-Stokes, whose reader takes the top
        // first (src/file_io.cpp:602-603 against 297-298)
        w.i4(s.bc_bot); w.i4(s.bc_top);
        w.i4(s.free_slip_bot); w.i4(s.free_slip_top);
        w.f8(s.bc_bot_flux); w.f8(s.bc_top_flux);
        w.put(s.p_constant.data(), 4 * nc);
        if (s.cfd_solver == 0) {
            w.f8(s.ns_gamma); w.f8(s.ns_theta); w.f8(s.ns_beta);
            w.f8(s.tolerance); w.u4(s.maxiter); w.u4(s.ndem);
            w.f8(s.c_phi); w.f8(s.c_v); w.f8(s.dt_dem_fac);
            for (const std::vector<d4> *a : {&s.f_d, &s.f_p, &s.f_v, &s.f_sum})
                for (uint32_t i = 0; i < n; ++i) w.put(&(*a)[i], 24);
        } else {
            w.f8(s.tolerance); w.u4(s.maxiter); w.u4(s.ndem); w.f8(s.c_phi);
            for (uint32_t i = 0; i < n; ++i) w.put(&s.f_p[i], 24);
            w.f8(s.beta_f); w.f8(s.k_c);
        }
    }
    w.put(s.color.data(), 4 * (size_t)n);
    return w.out;
}

int write_bin_file(const char *path, const HostState &s, std::string &err)
{
    std::vector<uint8_t> b = serialize_bin(s);
    FILE *f = std::fopen(path, "wb");
    if (!f) { err = std::string("could not create output binary file '") + path + "'"; return ST_FILE; }
    size_t put = std::fwrite(b.data(), 1, b.size(), f);
    std::fclose(f);
    if (put != b.size()) { err = "short write"; return ST_FILE; }
    return ST_OK;
}

static bool finite4(const d4 &v)
{
    return v.x == v.x && v.y == v.y && v.z == v.z && v.w == v.w;
}

int check_values(const HostState &s, std::string &err)
{
    char m[256];
    auto fail = [&](const char *msg) { err = msg; return ST_INPUT; };
    if (s.t_current > s.t_total || s.t_current < 0.0)
        return fail("the current time is outside [0, total]");
    if (s.origo[0] < 0.0 || s.origo[1] < 0.0 || s.origo[2] < 0.0)
        return fail("negative grid origo");
    if (s.L[0] <= 0.0 || s.L[1] <= 0.0 || s.L[2] <= 0.0)
        return fail("non-positive world size");
    if (s.num[0] == 0 || s.num[1] == 0 || s.num[2] == 0)
        return fail("zero grid cells along an axis");
    if (s.periodic == 2 && s.num[0] < 3)
        return fail("periodic x needs at least 3 cells along x");
    if (s.periodic == 1 && (s.num[0] < 3 || s.num[1] < 3))
        return fail("periodic x/y needs at least 3 cells along x and y");
    if (s.ncells() > 0xfffffffeull)
        return fail("more grid cells than 32-bit cell ids hold");
    for (uint32_t i = 0; i < s.np; ++i) {
        const d4 &x = s.x[i];
        if (x.w <= 0.0) {
            std::snprintf(m, sizeof m, "particle %u has a non-positive radius", i);
            err = m;
            return ST_INPUT;
        }
        if (!finite4(x) || !finite4(s.vel[i])) {
            std::snprintf(m, sizeof m, "particle %u has a NaN position or velocity", i);
            err = m;
            return ST_INPUT;
        }
        if (x.x < s.origo[0] || x.y < s.origo[1] || x.z < s.origo[2] ||
            x.x > s.L[0] || x.y > s.L[1] || x.z > s.L[2]) {
            std::snprintf(m, sizeof m, "particle %u is outside the grid", i);
            err = m;
            return ST_INPUT;
        }
    }
    if (s.nw > 0) {
        double z_max = 0.0;
        for (uint32_t i = 0; i < s.np; ++i)
            if (s.x[i].z > z_max) z_max = s.x[i].z;
        if (s.wnx[0].w < z_max) return fail("the upper wall is below the highest particle");
    }
    if (s.k_n <= 0.0) return fail("k_n must be positive");
    if (s.E < 0.0) return fail("E must not be negative");
    if (s.rho <= 0.0) return fail("rho must be positive");
    if (s.fluid && s.cfd_solver == 0) {
        // checkValues (src/sphere.cpp:311-317)
        if (s.rho_f <= 0.0) return fail("fluid density must be positive");
        // DEM::startTime reads the host pressure at cell (2,2,2)
        // (device.cu:1564), inside the grid only from 3 cells per axis
        if (s.num[0] < 3 || s.num[1] < 3 || s.num[2] < 3)
            return fail("the Navier-Stokes grid needs at least 3 cells per axis");
        if (s.ndem == 0) return fail("ndem must be positive");
    }
    if (s.fluid && s.cfd_solver == 1) {
        if (s.rho_f <= 0.0) return fail("fluid density must be positive");
        if (s.mu <= 0.0) return fail("fluid viscosity must be positive");
        if (s.beta_f <= 0.0) return fail("fluid compressibility must be positive");
        if (s.k_c <= 0.0) return fail("permeability prefactor must be positive");
    }
    for (uint32_t b = 0; b < s.nb0; ++b) {
        if (s.bonds[2 * b + 1] >= s.np || (s.bonds[2 * b] >= s.np && s.bonds[2 * b] != s.nb0 && s.bonds[2 * b] < s.np))
            return fail("bond refers to a particle index beyond np");
    }
    return ST_OK;
}

}  // namespace sphb
