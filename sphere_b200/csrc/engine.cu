// Engine orchestration and the C ABI (include/sphere_b200.h).
//
// Replaces the reference's DEM constructor, device set-up and time loop
// (src/sphere.cpp:16-95, src/device.cu:405-829 and :833-2834).  Steps run
// as CUDA graphs of `graph_steps` DEM steps; the loop counters live on the
// device so a captured graph replays unchanged.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/sphere_b200.h"
#include "dem_launch.h"
#include "engine_internal.h"
#include "host_state.h"

namespace sphb {

static thread_local std::string g_open_error;

// ---------------------------------------------------------------------
// permutation helpers
// ---------------------------------------------------------------------
template <class T>
__global__ void k_unsort(const T *src, T *dst, const uint32_t *orig_of, size_t np)
{
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k < np) dst[orig_of[k]] = src[k];
}
template <class T>
__global__ void k_sort_into(const T *src, T *dst, const uint32_t *orig_of, size_t np)
{
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k < np) dst[k] = src[orig_of[k]];
}

cudaError_t launch_unsort(const void *src, void *dst, const uint32_t *orig_of, size_t np,
                          size_t elem, cudaStream_t st)
{
    if (!np) return cudaSuccess;
    unsigned g = (unsigned)((np + 255) / 256);
    if (elem == 32) k_unsort<double4><<<g, 256, 0, st>>>((const double4 *)src, (double4 *)dst, orig_of, np);
    else if (elem == 8) k_unsort<double><<<g, 256, 0, st>>>((const double *)src, (double *)dst, orig_of, np);
    else if (elem == 4) k_unsort<uint32_t><<<g, 256, 0, st>>>((const uint32_t *)src, (uint32_t *)dst, orig_of, np);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_sort_into(const void *src, void *dst, const uint32_t *orig_of, size_t np,
                             size_t elem, cudaStream_t st)
{
    if (!np) return cudaSuccess;
    unsigned g = (unsigned)((np + 255) / 256);
    if (elem == 32) k_sort_into<double4><<<g, 256, 0, st>>>((const double4 *)src, (double4 *)dst, orig_of, np);
    else if (elem == 8) k_sort_into<double><<<g, 256, 0, st>>>((const double *)src, (double *)dst, orig_of, np);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------
Engine::~Engine()
{
    conv_close();
    darcy_free();
    ns_free();
    persist_free();
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (void *p : allocations) cudaFree(p);
    if (host_pinned) cudaFreeHost(host_pinned);
    if (stream) cudaStreamDestroy(stream);
}

int Engine::fail(int code, const std::string &msg)
{
    err = msg;
    return code;
}

int Engine::cuda_fail(cudaError_t e, const char *where)
{
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return ST_CUDA;
}


void Engine::build_params()
{
    const HostState &h = hs;
    DevParams &p = P;
    std::memset(&p, 0, sizeof p);
    p.np = h.np;
    p.nc = capacity;
    p.nw = h.nw;
    p.nb0 = h.nb0;
    p.ncells = (uint32_t)h.ncells();
    p.nblocks256 = (h.np + 255) / 256;
    for (int d = 0; d < 3; ++d) {
        p.num[d] = h.num[d];
        p.origo[d] = h.origo[d];
        p.L[d] = h.L[d];
        p.g[d] = h.g[d];
    }
    p.periodic = h.periodic;
    p.contactmodel = h.contactmodel;
    p.integrator = integrator;
    for (int w = 0; w < 6; ++w) p.wmode[w] = h.wmode[w];
    p.dt = h.dt;
    p.k_n = h.k_n; p.k_t = h.k_t; p.E = h.E; p.gamma_n = h.gamma_n; p.gamma_t = h.gamma_t;
    p.mu_s = h.mu_s; p.mu_d = h.mu_d; p.gamma_wn = h.gamma_wn; p.gamma_wt = h.gamma_wt;
    p.mu_ws = h.mu_ws; p.mu_wd = h.mu_wd; p.rho = h.rho;
    p.kappa = h.kappa; p.db = h.db; p.V_b = h.V_b;
    p.sigma0_A = h.sigma0_A; p.sigma0_f = h.sigma0_f; p.tau_x = h.tau_x;
    p.lambda_bar = h.lambda_bar; p.sigma_b = h.sigma_b; p.tau_b = h.tau_b;
    // neighbour-list skin: a tenth of the smallest radius
    double rmin = 1e300;
    for (uint32_t i = 0; i < h.np; ++i) rmin = std::min(rmin, h.x[i].w);
    p.skin = h.np ? 0.1 * rmin : 0.0;
    p.nlmax = nlmax;
    p.inject = inject;
}

int Engine::allocate_and_upload()
{
    const HostState &h = hs;
    size_t n = h.np;
    size_t slots = n * capacity;
    S.x = dalloc<double4>(n); S.vel = dalloc<double4>(n); S.angvel = dalloc<double4>(n);
    S.angpos = dalloc<double4>(n); S.acc = dalloc<double4>(n); S.angacc = dalloc<double4>(n);
    S.xyzsum = dalloc<double4>(n); S.force = dalloc<double4>(n); S.torque = dalloc<double4>(n);
    S.es_dot = dalloc<double>(n); S.es = dalloc<double>(n); S.ev_dot = dalloc<double>(n);
    S.ev = dalloc<double>(n); S.p = dalloc<double>(n);
    S.orig_of = dalloc<uint32_t>(n); S.pos_of = dalloc<uint32_t>(n);
    S.cell_of = dalloc<uint32_t>(n); S.cell_new = dalloc<uint32_t>(n);
    S.cell_start = dalloc<uint32_t>(h.ncells()); S.cell_end = dalloc<uint32_t>(h.ncells());
    S.contacts = dalloc<uint32_t>(slots); S.dmcode = dalloc<uint8_t>(slots);
    S.delta_t = dalloc<double4>(slots);
    S.occ = dalloc<uint64_t>(n);
    if (precision == SPH_PREC_MIXED) {
        S.vel_f = dalloc<float4>(n);
        S.angvel_f = dalloc<float4>(n);
        S.delta_t_f = dalloc<float4>(slots);
    }
    // the other buffer of the x / vel / angvel pair for the fused step paths
    if (fused_eligible() && step_kernel != 1 && step_kernel != 3) {
        S.x_nx = dalloc<double4>(n); S.vel_nx = dalloc<double4>(n); S.angvel_nx = dalloc<double4>(n);
        if (precision == SPH_PREC_MIXED) {
            S.vel_f_nx = dalloc<float4>(n);
            S.angvel_f_nx = dalloc<float4>(n);
        }
        if (!S.x_nx || !S.vel_nx || !S.angvel_nx) return fail(ST_CUDA, "device allocation failed");
    }
    S.nl = dalloc<uint32_t>(n * (size_t)nlmax);
    S.nl_count = dalloc<uint32_t>(n);
    S.x_ref = dalloc<float4>(n);
    S.wnx = dalloc<double4>(6); S.wmvfd = dalloc<double4>(6); S.wacc = dalloc<double>(6);
    S.walls_force_pp = dalloc<double>(n * (h.nw ? h.nw : 1));
    S.tau_pp = dalloc<double>(n);
    S.partials = dalloc<double>(P.nblocks256 + 1);
    S.tau_partials = dalloc<double>(P.nblocks256 + 1);
    S.bonds = dalloc<uint2>(h.nb0); S.bonds_delta = dalloc<double4>(h.nb0);
    S.bonds_omega = dalloc<double4>(h.nb0);
    S.bond_ptr = dalloc<uint32_t>(n + 1);
    S.count = dalloc<uint32_t>(h.ncells()); S.fill = dalloc<uint32_t>(h.ncells());
    S.vals = dalloc<uint32_t>(n);
    S.block_sums = dalloc<uint32_t>(4096);
    S.perm_scratch = dalloc<unsigned char>(resort_scratch_bytes(n));
    S.ctl = dalloc<DevCtl>(1);
    bond_f = dalloc<double4>(h.nb0);
    bond_t = dalloc<double4>(h.nb0);
    tmp = dalloc<unsigned char>(std::max<size_t>(slots * 32, n * 32) + 64);
    if (alloc_failed) return fail(ST_CUDA, "device allocation failed");

    // bonds: CSR of (bond << 1 | side) per particle, bonds in increasing order
    std::vector<uint32_t> ptr(n + 1, 0), list;
    for (uint32_t b = 0; b < h.nb0; ++b) {
        uint32_t i = h.bonds[2 * b], j = h.bonds[2 * b + 1];
        if (i < n) ptr[i + 1]++;
        if (j < n && i < n) ptr[j + 1]++;
    }
    for (size_t i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
    list.assign(ptr[n] ? ptr[n] : 1, 0);
    {
        std::vector<uint32_t> fillp(ptr.begin(), ptr.end() - 1);
        for (uint32_t b = 0; b < h.nb0; ++b) {
            uint32_t i = h.bonds[2 * b], j = h.bonds[2 * b + 1];
            if (i >= n) continue;  // erased before the run started
            list[fillp[i]++] = b << 1;
            if (j < n) list[fillp[j]++] = (b << 1) | 1;
        }
    }
    S.bond_list = dalloc<uint32_t>(list.size());

    // upload in original order: sorted storage starts as the identity
    auto up = [&](void *dst, const void *src, size_t bytes) {
        if (bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    };
    std::vector<double4> buf(n);
    auto up4 = [&](double4 *dst, const std::vector<d4> &src, bool zero_w) {
        for (size_t i = 0; i < n; ++i)
            buf[i] = make_double4(src[i].x, src[i].y, src[i].z, zero_w ? 0.0 : src[i].w);
        up(dst, buf.data(), n * 32);
        cudaStreamSynchronize(stream);
    };
    up4(S.x, h.x, false);
    up4(S.vel, h.vel, false);
    up4(S.angvel, h.angvel, true);
    up4(S.angpos, h.angpos, true);
    up4(S.xyzsum, h.xyzsum, true);
    up4(S.force, h.force, true);
    up4(S.torque, h.torque, true);
    up(S.es_dot, h.es_dot.data(), n * 8); up(S.es, h.es.data(), n * 8);
    up(S.ev_dot, h.ev_dot.data(), n * 8); up(S.ev, h.ev.data(), n * 8);
    up(S.p, h.p.data(), n * 8);
    std::vector<uint32_t> ident(n);
    for (size_t i = 0; i < n; ++i) ident[i] = (uint32_t)i;
    up(S.orig_of, ident.data(), n * 4);
    up(S.pos_of, ident.data(), n * 4);
    std::vector<uint32_t> empty(slots, (uint32_t)n);
    up(S.contacts, empty.data(), slots * 4);
    std::vector<double4> w4(6);
    for (int w = 0; w < 6; ++w) w4[w] = make_double4(h.wnx[w].x, h.wnx[w].y, h.wnx[w].z, h.wnx[w].w);
    up(S.wnx, w4.data(), 6 * 32);
    cudaStreamSynchronize(stream);
    for (int w = 0; w < 6; ++w) w4[w] = make_double4(h.wmvfd[w].x, h.wmvfd[w].y, h.wmvfd[w].z, h.wmvfd[w].w);
    up(S.wmvfd, w4.data(), 6 * 32);
    up(S.bonds, h.bonds.data(), h.nb0 * 8);
    std::vector<double4> bd(h.nb0), bo(h.nb0);
    for (uint32_t b = 0; b < h.nb0; ++b) {
        bd[b] = make_double4(h.bonds_delta[b].x, h.bonds_delta[b].y, h.bonds_delta[b].z, h.bonds_delta[b].w);
        bo[b] = make_double4(h.bonds_omega[b].x, h.bonds_omega[b].y, h.bonds_omega[b].z, h.bonds_omega[b].w);
    }
    up(S.bonds_delta, bd.data(), h.nb0 * 32);
    up(S.bonds_omega, bo.data(), h.nb0 * 32);
    up(S.bond_ptr, ptr.data(), (n + 1) * 4);
    up(S.bond_list, list.data(), list.size() * 4);
    DevCtl c;
    std::memset(&c, 0, sizeof c);
    c.iter = 0;
    c.t_current = h.t_current;
    c.velocity_state = 1;
    c.nl_rebuild = 1;
    up(S.ctl, &c, sizeof c);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload");
    host_t = h.t_current;
    host_iter = 0;
    // initial sort (the reference sorts at the start of every step)
    if ((e = launch_hash(P, S, stream)) != cudaSuccess) return cuda_fail(e, "hash");
    if ((e = launch_resort(P, S, S.perm_scratch, 1, stream)) != cudaSuccess) return cuda_fail(e, "sort");
    if ((e = launch_refresh_f(P, S, stream)) != cudaSuccess) return cuda_fail(e, "sort");
    return poll_errors("initial sort");
}

int Engine::poll_errors(const char *where)
{
    DevCtl c;
    cudaError_t e = cudaMemcpyAsync(&c, S.ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, where);
    last_ctl = c;
    if (c.err == DERR_NONE) return ST_OK;
    char m[256];
    switch (c.err) {
    case DERR_OUTSIDE:
        std::snprintf(m, sizeof m, "%s: particle %d moved outside the grid or became non-finite "
                      "(is the time step too large?)", where, c.err_index);
        err = m;
        return ST_OUTSIDE;
    case DERR_CAPACITY:
        std::snprintf(m, sizeof m, "%s: particle %d has more contacts than the %u slots per particle",
                      where, c.err_index, capacity);
        err = m;
        return ST_CAPACITY;
    case DERR_TIMEOUT:
        err = std::string(where) + ": a bounded device wait timed out";
        return ST_TIMEOUT;
    case DERR_BOND:
        std::snprintf(m, sizeof m, "%s: bond %d refers to a particle index beyond np", where, c.err_index);
        err = m;
        return ST_INPUT;
    default:
        std::snprintf(m, sizeof m, "%s: device error %d", where, c.err);
        err = m;
        return ST_CUDA;
    }
}

cudaError_t Engine::enqueue_stage(int stage)
{
    const int prec = precision == 0 ? 0 : 1;
    switch (stage) {
    case 0: return launch_resort(P, S, S.perm_scratch, 0, stream, 1);
    case 1:
        if (fused) {
            if (precision == SPH_PREC_MIXED) return launch_contacts_integrate_mixed(P, S, stream);
            return launch_contacts_integrate(P, S, prec, stream);
        }
        if (precision == SPH_PREC_MIXED)
            return launch_contacts_mixed(P, S, stream, step_kernel == 3);
        return launch_contacts(P, S, prec, stream, step_kernel == 3);
    case 2: return launch_bonds(P, S, prec, bond_f, bond_t, stream);
    case 3: return enqueue_fluid();
    case 4:
        if (fused) {
            // the step's integration went to the other buffer: it is current now
            cudaError_t e = launch_walls_step(P, S, stream);
            flip_view();
            return e;
        }
        return launch_integrate(P, S, stream);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t Engine::enqueue_step()
{
    for (int st = 0; st < 5; ++st) {
        cudaError_t e = enqueue_stage(st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int Engine::profile(uint64_t n, sph_profile *out)
{
    std::memset(out, 0, sizeof *out);
    cudaEvent_t ev[6];
    for (auto &x : ev) cudaEventCreate(&x);
    double ms[5] = {0, 0, 0, 0, 0}, total = 0;
    int rc = ST_OK;
    for (uint64_t i = 0; i < n && rc == ST_OK; ++i) {
        cudaEventRecord(ev[0], stream);
        for (int st = 0; st < 5; ++st) {
            cudaError_t e = enqueue_stage(st);
            if (e != cudaSuccess) { rc = cuda_fail(e, "profile"); break; }
            cudaEventRecord(ev[st + 1], stream);
        }
        if (rc) break;
        cudaEventSynchronize(ev[5]);
        for (int st = 0; st < 5; ++st) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[st], ev[st + 1]);
            ms[st] += t;
        }
        float t = 0;
        cudaEventElapsedTime(&t, ev[0], ev[5]);
        total += t;
        advance_host_clock(1);
        warmed = true;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    double inv = n ? 1.0 / (double)n : 0.0;
    out->resort_ms = ms[0] * inv;
    out->contacts_ms = ms[1] * inv;
    out->bonds_ms = ms[2] * inv;
    out->fluid_ms = ms[3] * inv;
    out->integrate_ms = ms[4] * inv;
    out->step_ms = total * inv;
    out->steps = n;
    return poll_errors("profile");
}

int Engine::ensure_graph()
{
    // kernels capture the state view by value: a graph made for the other
    // view (the persistent path flips views) is stale
    if (graph_exec && (graph_view != cur_view || graph_fused != fused)) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    if (graph_exec || graph_steps <= 1 || graph_failed) return ST_OK;
    graph_view = cur_view;
    graph_fused = fused;
    graph_exec = capture_steps(graph_len());
    if (!graph_exec) graph_failed = true;
    return ST_OK;
}

// A CUDA graph of k per-stage DEM steps on the current state view, or null
// when capture or instantiation fails (the caller then steps eagerly).
cudaGraphExec_t Engine::capture_steps(int k)
{
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    const int view0 = cur_view;   // fused steps flip the view while they are captured
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { cudaGetLastError(); return nullptr; }
    for (int i = 0; i < k && e == cudaSuccess; ++i) e = enqueue_step();
    cudaError_t e2 = cudaStreamEndCapture(stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        cur_view = view0;
        S = S_view[cur_view];
        return nullptr;
    }
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { cudaGetLastError(); return nullptr; }
    return x;
}

int Engine::step(uint64_t n)
{
    if (n == 0) return ST_OK;
    if (persist && !persist_off) return step_persistent(n);
    return step_stages(n);
}

// The per-stage kernels, replayed from a CUDA graph of graph_steps steps.
int Engine::step_stages(uint64_t n)
{
    if (n == 0) return ST_OK;
    if (!warmed) {
        // one eager step first: sets kernel attributes outside any capture
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "step");
        warmed = true;
        advance_host_clock(1);
        --n;
        int rc = poll_errors("step");
        if (rc) return rc;
    }
    ensure_graph();
    uint64_t done = 0;
    const uint64_t glen = (uint64_t)graph_len();
    while (graph_exec && n - done >= glen) {
        cudaError_t e = cudaGraphLaunch(graph_exec, stream);
        if (e != cudaSuccess) return cuda_fail(e, "graph launch");
        done += glen;
    }
    for (; done < n; ++done) {
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "step");
    }
    advance_host_clock(n);
    return poll_errors("step");
}

void Engine::advance_host_clock(uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) {
        host_t += hs.dt;
        filetimeclock += hs.dt;
        ++host_iter;
    }
}

// ----- field access -----
int64_t Engine::field_bytes(int f) const
{
    size_t n = hs.np, slots = n * capacity;
    switch (f) {
    case SPH_F_X: case SPH_F_VEL: case SPH_F_ANGVEL: case SPH_F_ANGPOS: case SPH_F_FORCE:
    case SPH_F_TORQUE: case SPH_F_ACC: case SPH_F_ANGACC: case SPH_F_XYZSUM:
        return (int64_t)n * 32;
    case SPH_F_ES_DOT: case SPH_F_ES: case SPH_F_EV_DOT: case SPH_F_EV: case SPH_F_P:
        return (int64_t)n * 8;
    case SPH_F_CELLID: case SPH_F_INDEX: return (int64_t)n * 4;
    case SPH_F_CELLSTART: case SPH_F_CELLEND: return (int64_t)hs.ncells() * 4;
    case SPH_F_CONTACTS: return (int64_t)slots * 4;
    case SPH_F_DELTA_T: case SPH_F_DISTMOD: return (int64_t)slots * 32;
    case SPH_F_WALLS_NX: case SPH_F_WALLS_MVFD: return (int64_t)hs.nw * 32;
    case SPH_F_WALLS_ACC: return (int64_t)hs.nw * 8;
    case SPH_F_ITER: case SPH_F_VELOCITY_STATE: return 8;
    case SPH_F_TIME: return 8;
    case SPH_F_BONDS: return (int64_t)hs.nb0 * 8;
    case SPH_F_BONDS_DELTA: case SPH_F_BONDS_OMEGA: return (int64_t)hs.nb0 * 32;
    default: return darcy_field_bytes(f);
    }
}

double4 *Engine::sorted_vec(int f) const
{
    switch (f) {
    case SPH_F_X: return S.x; case SPH_F_VEL: return S.vel; case SPH_F_ANGVEL: return S.angvel;
    case SPH_F_ANGPOS: return S.angpos; case SPH_F_FORCE: return S.force;
    case SPH_F_TORQUE: return S.torque; case SPH_F_ACC: return S.acc;
    case SPH_F_ANGACC: return S.angacc; case SPH_F_XYZSUM: return S.xyzsum;
    default: return nullptr;
    }
}

double *Engine::sorted_scalar(int f) const
{
    switch (f) {
    case SPH_F_ES_DOT: return S.es_dot; case SPH_F_ES: return S.es;
    case SPH_F_EV_DOT: return S.ev_dot; case SPH_F_EV: return S.ev; case SPH_F_P: return S.p;
    default: return nullptr;
    }
}

int Engine::get(int f, void *dst, size_t bytes)
{
    int64_t need = field_bytes(f);
    if (need < 0) return fail(ST_ARG, "unknown field");
    if ((!dst && need > 0) || bytes < (size_t)need) return fail(ST_ARG, "destination buffer too small");
    size_t n = hs.np;
    cudaError_t e = cudaSuccess;
    auto d2h = [&](const void *src, size_t b) {
        if (b) e = cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, stream);
    };
    if (double4 *src = sorted_vec(f)) {
        e = launch_unsort(src, tmp, S.orig_of, n, 32, stream);
        d2h(tmp, n * 32);
    } else if (double *src = sorted_scalar(f)) {
        e = launch_unsort(src, tmp, S.orig_of, n, 8, stream);
        d2h(tmp, n * 8);
    } else {
        switch (f) {
        case SPH_F_CELLID: d2h(S.cell_of, n * 4); break;
        case SPH_F_INDEX: d2h(S.orig_of, n * 4); break;
        case SPH_F_CELLSTART: d2h(S.cell_start, (size_t)need); break;
        case SPH_F_CELLEND: d2h(S.cell_end, (size_t)need); break;
        case SPH_F_CONTACTS: d2h(S.contacts, (size_t)need); break;
        case SPH_F_DELTA_T:
            if (S.delta_t_f) return get_delta_t_mixed((double *)dst);
            d2h(S.delta_t, (size_t)need);
            break;
        case SPH_F_DISTMOD: return get_distmod((double *)dst);
        case SPH_F_WALLS_NX: d2h(S.wnx, (size_t)need); break;
        case SPH_F_WALLS_MVFD: d2h(S.wmvfd, (size_t)need); break;
        case SPH_F_WALLS_ACC: d2h(S.wacc, (size_t)need); break;
        case SPH_F_ITER: {
            int rc = poll_errors("get");
            if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
            std::memcpy(dst, &last_ctl.iter, 8);
            return ST_OK;
        }
        case SPH_F_TIME: {
            int rc = poll_errors("get");
            if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
            std::memcpy(dst, &last_ctl.t_current, 8);
            return ST_OK;
        }
        case SPH_F_VELOCITY_STATE: {
            int rc = poll_errors("get");
            if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
            int64_t v = last_ctl.velocity_state;
            std::memcpy(dst, &v, 8);
            return ST_OK;
        }
        case SPH_F_BONDS: d2h(S.bonds, (size_t)need); break;
        case SPH_F_BONDS_DELTA: d2h(S.bonds_delta, (size_t)need); break;
        case SPH_F_BONDS_OMEGA: d2h(S.bonds_omega, (size_t)need); break;
        default: return darcy_get(f, dst, bytes);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "get");
    return ST_OK;
}

int Engine::get_distmod(double *dst)
{
    size_t n = hs.np, slots = n * capacity;
    std::vector<uint32_t> c(slots);
    std::vector<uint8_t> code(slots);
    std::vector<double> xs(n * 4);
    cudaMemcpyAsync(c.data(), S.contacts, slots * 4, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(code.data(), S.dmcode, slots, cudaMemcpyDeviceToHost, stream);
    int rc = get(SPH_F_X, xs.data(), xs.size() * 8);
    if (rc) return rc;
    for (size_t s = 0; s < slots; ++s) {
        double *o = dst + 4 * s;
        o[0] = o[1] = o[2] = o[3] = 0.0;
        if (c[s] >= n) continue;
        double dx = 0.0, dy = 0.0;
        if (code[s] & 1) dx = dx + hs.L[0];
        if (code[s] & 2) dx = dx - hs.L[0];
        if (code[s] & 4) dy = dy + hs.L[1];
        if (code[s] & 8) dy = dy - hs.L[1];
        o[0] = dx; o[1] = dy; o[2] = 0.0; o[3] = xs[4 * c[s] + 3];
    }
    return ST_OK;
}

int Engine::get_delta_t_mixed(double *dst)
{
    size_t slots = (size_t)hs.np * capacity;
    std::vector<float4> f(slots);
    cudaError_t e = cudaMemcpyAsync(f.data(), S.delta_t_f, slots * 16, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "get");
    for (size_t i = 0; i < slots; ++i) {
        dst[4 * i] = f[i].x; dst[4 * i + 1] = f[i].y; dst[4 * i + 2] = f[i].z; dst[4 * i + 3] = 0.0;
    }
    return ST_OK;
}

int Engine::set(int f, const void *src, size_t bytes)
{
    int64_t need = field_bytes(f);
    if (need < 0 || bytes != (size_t)need) return fail(ST_ARG, "source size does not match the field");
    size_t n = hs.np;
    cudaError_t e = cudaSuccess;
    if (double4 *dst = sorted_vec(f)) {
        e = cudaMemcpyAsync(tmp, src, n * 32, cudaMemcpyHostToDevice, stream);
        // positions: the next step re-sorts and rebuilds the lists where
        // they changed (k_set_positions raises the flags)
        if (e == cudaSuccess && f == SPH_F_X) e = launch_set_positions(P, S, (const double4 *)tmp, stream);
        else if (e == cudaSuccess) e = launch_sort_into(tmp, dst, S.orig_of, n, 32, stream);
    } else if (double *dst = sorted_scalar(f)) {
        e = cudaMemcpyAsync(tmp, src, n * 8, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = launch_sort_into(tmp, dst, S.orig_of, n, 8, stream);
    } else {
        switch (f) {
        case SPH_F_CONTACTS:
            e = cudaMemcpyAsync(S.contacts, src, bytes, cudaMemcpyHostToDevice, stream);
            if (e == cudaSuccess) e = launch_occ_from_rows(P, S, stream);
            break;
        case SPH_F_DELTA_T:
            if (S.delta_t_f) {
                std::vector<float4> f(bytes / 32);
                const double *d = (const double *)src;
                for (size_t i = 0; i < f.size(); ++i)
                    f[i] = make_float4((float)d[4 * i], (float)d[4 * i + 1], (float)d[4 * i + 2], 0.f);
                e = cudaMemcpyAsync(S.delta_t_f, f.data(), f.size() * 16, cudaMemcpyHostToDevice, stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            } else {
                e = cudaMemcpyAsync(S.delta_t, src, bytes, cudaMemcpyHostToDevice, stream);
            }
            break;
        case SPH_F_WALLS_NX: e = cudaMemcpyAsync(S.wnx, src, bytes, cudaMemcpyHostToDevice, stream); break;
        case SPH_F_WALLS_MVFD: e = cudaMemcpyAsync(S.wmvfd, src, bytes, cudaMemcpyHostToDevice, stream); break;
        case SPH_F_WALLS_ACC: e = cudaMemcpyAsync(S.wacc, src, bytes, cudaMemcpyHostToDevice, stream); break;
        case SPH_F_DISTMOD: {
            // (dx, dy, 0, r_partner) per slot -> the periodic shift code
            const double *d = (const double *)src;
            std::vector<uint8_t> code(bytes / 32);
            for (size_t i = 0; i < code.size(); ++i) {
                const double dx = d[4 * i], dy = d[4 * i + 1];
                code[i] = (uint8_t)((dx > 0.0 ? 1 : 0) | (dx < 0.0 ? 2 : 0) | (dy > 0.0 ? 4 : 0) |
                                    (dy < 0.0 ? 8 : 0));
            }
            e = cudaMemcpyAsync(S.dmcode, code.data(), code.size(), cudaMemcpyHostToDevice, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            break;
        }
        case SPH_F_ITER: case SPH_F_VELOCITY_STATE: {
            // loop state: DevCtl on the device, the host mirror of the counter
            int rc = poll_errors("set");
            if (rc < 0) return rc;
            int64_t v;
            std::memcpy(&v, src, 8);
            if (f == SPH_F_ITER) {
                if (v < 0) return fail(ST_ARG, "iter must not be negative");
                long long it = (long long)v;
                e = cudaMemcpyAsync(&S.ctl->iter, &it, sizeof it, cudaMemcpyHostToDevice, stream);
                host_iter = v;
            } else {
                int vs = (int)v;
                e = cudaMemcpyAsync(&S.ctl->velocity_state, &vs, sizeof vs, cudaMemcpyHostToDevice, stream);
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            break;
        }
        default: return fail(ST_ARG, "field is read-only");
        }
    }
    // the FP32 velocity copies of the mixed mode follow the FP64 velocities
    if (e == cudaSuccess && (f == SPH_F_VEL || f == SPH_F_ANGVEL)) e = launch_refresh_f(P, S, stream);
    if (e != cudaSuccess) return cuda_fail(e, "set");
    return poll_errors("set");   // waits for the copies out of the caller's buffer
}

int Engine::download_state()
{
    size_t n = hs.np;
    std::vector<double4> b4(n);
    auto get4 = [&](int f, std::vector<d4> &dst) {
        int rc = get(f, b4.data(), n * 32);
        if (rc) return rc;
        for (size_t i = 0; i < n; ++i) {
            dst[i].x = b4[i].x; dst[i].y = b4[i].y; dst[i].z = b4[i].z;
            if (f == SPH_F_X || f == SPH_F_VEL) dst[i].w = b4[i].w;
        }
        return 0;
    };
    int rc;
    if ((rc = get4(SPH_F_X, hs.x)) || (rc = get4(SPH_F_VEL, hs.vel)) ||
        (rc = get4(SPH_F_ANGVEL, hs.angvel)) || (rc = get4(SPH_F_ANGPOS, hs.angpos)) ||
        (rc = get4(SPH_F_FORCE, hs.force)) || (rc = get4(SPH_F_TORQUE, hs.torque)) ||
        (rc = get4(SPH_F_XYZSUM, hs.xyzsum)))
        return rc;
    if ((rc = get(SPH_F_ES_DOT, hs.es_dot.data(), n * 8)) || (rc = get(SPH_F_ES, hs.es.data(), n * 8)) ||
        (rc = get(SPH_F_EV_DOT, hs.ev_dot.data(), n * 8)) || (rc = get(SPH_F_EV, hs.ev.data(), n * 8)) ||
        (rc = get(SPH_F_P, hs.p.data(), n * 8)))
        return rc;
    std::vector<double4> w(6);
    cudaMemcpyAsync(w.data(), S.wnx, 6 * 32, cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    for (uint32_t i = 0; i < hs.nw; ++i) hs.wnx[i] = d4{w[i].x, w[i].y, w[i].z, w[i].w};
    cudaMemcpyAsync(w.data(), S.wmvfd, 6 * 32, cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    for (uint32_t i = 0; i < hs.nw; ++i) hs.wmvfd[i] = d4{w[i].x, w[i].y, w[i].z, w[i].w};
    if (hs.nb0) {
        cudaMemcpyAsync(hs.bonds.data(), S.bonds, hs.nb0 * 8, cudaMemcpyDeviceToHost, stream);
        std::vector<double4> bd(hs.nb0), bo(hs.nb0);
        cudaMemcpyAsync(bd.data(), S.bonds_delta, hs.nb0 * 32, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(bo.data(), S.bonds_omega, hs.nb0 * 32, cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        for (uint32_t b = 0; b < hs.nb0; ++b) {
            hs.bonds_delta[b] = d4{bd[b].x, bd[b].y, bd[b].z, bd[b].w};
            hs.bonds_omega[b] = d4{bo[b].x, bo[b].y, bo[b].z, bo[b].w};
        }
    }
    rc = darcy_download();
    if (rc) return rc;
    rc = poll_errors("download");
    hs.t_current = last_ctl.t_current;
    return rc;
}

// Writing a file also refreshes the host's copy of wall 0 that the Darcy
// solver reads and restarts the file clock (device.cu:2556-2600).
int Engine::write_bin(const char *path)
{
    int rc = download_state();
    if (rc < 0) return rc;
    filetimeclock = 0.0;
    ns_set_host_wall();
    if (darcy) {
        darcy_set_host_wall();
        if ((rc = darcy_sync_wall()) < 0) return rc;
    }
    return write_bin_file(path, hs, err);
}

int Engine::write_status()
{
    std::string f = outdir + "/" + sid + ".status.dat";
    FILE *fp = std::fopen(f.c_str(), "w");
    if (!fp) return fail(ST_FILE, "could not write " + f);
    std::fprintf(fp, "%2.4e %2.4e %d\n", hs.t_current, 100.0 * hs.t_current / hs.t_total,
                 hs.step_count);
    std::fclose(fp);
    return ST_OK;
}

// DEM::startTime's loop control (device.cu:845-2684) with file output.
int Engine::run()
{
    char name[512];
    int rc;
    if (hs.step_count == 0) {
        std::snprintf(name, sizeof name, "%s/%s.output00000.bin", outdir.c_str(), sid.c_str());
        if ((rc = write_bin(name)) < 0) return rc;
    }
    hs.t_current = host_t;
    if ((rc = write_status()) < 0) return rc;
    conv_open();
    double t = host_t;
    int warn = ST_OK;
    while (t <= hs.t_total) {
        // steps until the next file output or the end of the run
        uint64_t n = 0;
        bool output = false;
        double tt = t, fc = filetimeclock;
        while (tt <= hs.t_total) {
            tt += hs.dt;
            fc += hs.dt;
            ++n;
            if (fc >= hs.file_dt) { output = true; break; }
        }
        if ((rc = step_with_fluid_log(n)) < 0) return rc;
        if (rc > 0) warn = rc;
        t = tt;
        if (output) {
            // the Navier-Stokes stability check precedes each file
            // (device.cu:2612-2616)
            if (ns && ((rc = download_state()) < 0 || (rc = ns_check_stability()) < 0)) return rc;
            hs.step_count += 1;
            std::snprintf(name, sizeof name, "%s/%s.output%05d.bin", outdir.c_str(), sid.c_str(),
                          hs.step_count);
            if ((rc = write_bin(name)) < 0) return rc;
            hs.t_current = t;
            if ((rc = write_status()) < 0) return rc;
        }
        if (verbose)
            std::printf("\r  Current time: %g/%g s.      ", t, hs.t_total);
    }
    if (verbose) std::printf("\n");
    conv_close();
    return warn;
}

}  // namespace sphb

static_assert(sphb::kInjectResort == SPH_INJECT_RESORT && sphb::kInjectPersistent == SPH_INJECT_PERSISTENT &&
                  sphb::kInjectDarcy == SPH_INJECT_DARCY && sphb::kInjectNS == SPH_INJECT_NS,
              "fault-injection bits of the device code and the C ABI");

using sphb::Engine;

struct sph_engine {
    std::unique_ptr<Engine> e;
};

extern "C" {

int sph_default_opts(sph_opts *o)
{
    // the caller's struct_size is read before anything is written: a caller
    // compiled against another layout gets an error, not an overwrite
    if (!o || o->struct_size != sizeof(sph_opts)) return SPH_ERR_ARG;
    std::memset(o, 0, sizeof *o);
    o->struct_size = sizeof(sph_opts);
    o->device = -1;
    o->precision = SPH_PREC_FAITHFUL;
    o->integrator = 3;
    o->contact_capacity = 32;
    o->graph_steps = 0;
    return SPH_OK;
}

static int open_common(std::unique_ptr<Engine> &eng, const sph_opts *opts)
{
    sph_opts o;
    if (opts) {
        o = *opts;
    } else {
        o.struct_size = sizeof(sph_opts);
        sph_default_opts(&o);
    }
    Engine &e = *eng;
    e.precision = o.precision;
    e.integrator = o.integrator == 2 ? 2 : 3;
    e.capacity = o.contact_capacity > 0 ? (uint32_t)o.contact_capacity : 32;
    if (e.capacity > 64)
        return e.fail(sphb::ST_ARG, "contact_capacity above 64 slots is not supported");
    if (e.hs.np >= (1u << 28))
        return e.fail(sphb::ST_UNSUPPORTED, "more than 2^28 particles");
    e.verbose = o.verbose;
    e.graph_steps = o.graph_steps > 0 ? o.graph_steps : 64;
    e.warm_start = o.warm_start;
    e.step_kernel = o.step_kernel;
    e.darcy_exact_stop = o.darcy_exact_stop ? 1 : 0;
    e.inject = (uint32_t)o.inject_timeout;
    e.outdir = o.output_dir ? o.output_dir : "output";
    if (e.step_kernel < 0 || e.step_kernel > 4) return e.fail(sphb::ST_ARG, "unknown step_kernel");
    if (e.precision != SPH_PREC_FAITHFUL && e.precision != SPH_PREC_FP64 &&
        e.precision != SPH_PREC_MIXED)
        return e.fail(sphb::ST_ARG, "unknown precision mode");
    if (e.hs.contactmodel == 3)
        return e.fail(sphb::ST_UNSUPPORTED,
                      "contact model 3 (Hertz-Mindlin) is not built: the reference's contactHertz "
                      "takes powers of the negative overlap and returns NaN forces for every contact");
    if (e.hs.contactmodel != 1 && e.hs.contactmodel != 2)
        return e.fail(sphb::ST_INPUT, "contact model not understood");
    int rc = sphb::check_values(e.hs, e.err);
    if (rc) return rc;
    if (o.device >= 0) {
        cudaError_t ce = cudaSetDevice(o.device);
        if (ce != cudaSuccess) return e.cuda_fail(ce, "cudaSetDevice");
    }
    cudaError_t ce = cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return e.cuda_fail(ce, "cudaStreamCreate");
    e.build_params();
    if (e.precision == SPH_PREC_MIXED) {
        rc = e.mixed_init();
        if (rc) return rc;
    }
    if (e.step_kernel == 2 && !e.persist_eligible())
        return e.fail(sphb::ST_UNSUPPORTED, "the fused step kernel does not cover bonds, fluid or "
                                            "the shear-stress wall (wmode 3)");
    if (e.step_kernel == 4 && !e.fused_eligible())
        return e.fail(sphb::ST_UNSUPPORTED, "contacts and integration in one launch do not cover "
                                            "bonds, fluid or the shear-stress wall (wmode 3)");
    e.fused = e.step_kernel == 4;
    rc = e.allocate_and_upload();
    if (rc) return rc;
    rc = e.darcy_init();
    if (rc) return rc;
    e.make_views();
    return e.persist_init();
}

static std::string sid_from_path(const char *path)
{
    std::string s(path);
    size_t slash = s.rfind('/');
    size_t start = slash == std::string::npos ? 0 : slash + 1;
    size_t dot = s.rfind('.');
    if (dot == std::string::npos || dot < start) dot = s.size();
    return s.substr(start, dot - start);
}

int sph_open(const char *bin_path, const sph_opts *opts, sph_engine **out)
{
    if (!bin_path || !out) return SPH_ERR_ARG;
    *out = nullptr;
    if (opts && opts->struct_size != sizeof(sph_opts)) {
        sphb::g_open_error = "sph_opts.struct_size does not match this library's sph_opts";
        return SPH_ERR_ARG;
    }
    auto eng = std::make_unique<Engine>();
    int fluid = opts ? opts->fluid : 0;
    int rc = sphb::read_bin_file(bin_path, fluid, eng->hs, eng->err);
    if (rc == 0) {
        eng->sid = sid_from_path(bin_path);
        rc = open_common(eng, opts);
    }
    if (rc < 0) {
        sphb::g_open_error = eng->err;
        return rc;
    }
    *out = new sph_engine{std::move(eng)};
    return rc;
}

int sph_open_buffer(const void *bytes, size_t nbytes, const sph_opts *opts, const char *sid,
                    sph_engine **out)
{
    if (!bytes || !out) return SPH_ERR_ARG;
    *out = nullptr;
    if (opts && opts->struct_size != sizeof(sph_opts)) {
        sphb::g_open_error = "sph_opts.struct_size does not match this library's sph_opts";
        return SPH_ERR_ARG;
    }
    auto eng = std::make_unique<Engine>();
    int fluid = opts ? opts->fluid : 0;
    int rc = sphb::parse_bin((const uint8_t *)bytes, nbytes, fluid, eng->hs, eng->err);
    if (rc == 0) {
        eng->sid = sid ? sid : "unnamed";
        rc = open_common(eng, opts);
    }
    if (rc < 0) {
        sphb::g_open_error = eng->err;
        return rc;
    }
    *out = new sph_engine{std::move(eng)};
    return rc;
}

const char *sph_open_error(void) { return sphb::g_open_error.c_str(); }

}  // extern "C"

namespace sphb {

// Opens one engine from a file path or from the bytes of a .bin file (the
// batch engine opens its boxes with this).
int open_engine(const char *path, const void *bytes, size_t nbytes, const sph_opts *opts,
                const char *sid, std::unique_ptr<Engine> &out, std::string &err)
{
    if (opts && opts->struct_size != sizeof(sph_opts)) {
        err = "sph_opts.struct_size does not match this library's sph_opts";
        return SPH_ERR_ARG;
    }
    auto eng = std::make_unique<Engine>();
    int fluid = opts ? opts->fluid : 0;
    int rc = path ? read_bin_file(path, fluid, eng->hs, eng->err)
                  : parse_bin((const uint8_t *)bytes, nbytes, fluid, eng->hs, eng->err);
    if (rc == 0) {
        eng->sid = path ? sid_from_path(path) : (sid ? sid : "unnamed");
        rc = open_common(eng, opts);
    }
    if (rc < 0) {
        err = eng->err;
        return rc;
    }
    out = std::move(eng);
    return rc;
}

}  // namespace sphb

extern "C" {

int sph_check_file(const char *bin_path, int fluid)
{
    if (!bin_path) return SPH_ERR_ARG;
    sphb::HostState hs;
    std::string err;
    int rc = sphb::read_bin_file(bin_path, fluid, hs, err);
    if (rc == 0 && hs.contactmodel != 1 && hs.contactmodel != 2 && hs.contactmodel != 3) {
        err = "contact model not understood";
        rc = SPH_ERR_INPUT;
    }
    if (rc == 0) rc = sphb::check_values(hs, err);
    sphb::g_open_error = rc ? err : std::string();
    return rc;
}

int sph_run(sph_engine *e) { return e ? e->e->run() : SPH_ERR_ARG; }

int sph_profile_steps(sph_engine *e, uint64_t n, sph_profile *out)
{
    return (e && out) ? e->e->profile(n, out) : SPH_ERR_ARG;
}

int sph_step(sph_engine *e, uint64_t n) { return e ? e->e->step_with_fluid_log(n) : SPH_ERR_ARG; }

int sph_step_timed(sph_engine *e, uint64_t n, double *device_ms)
{
    if (!e || !device_ms) return SPH_ERR_ARG;
    Engine &g = *e->e;
    if (!g.warmed && n > 0) {
        int rc = g.step_with_fluid_log(1);
        if (rc < 0) return rc;
        --n;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, g.stream);
    int rc = g.step_with_fluid_log(n);
    cudaEventRecord(b, g.stream);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *device_ms = ms;
    return rc;
}

int64_t sph_field_bytes(sph_engine *e, sph_field f)
{
    if (!e) return SPH_ERR_ARG;
    int64_t b = e->e->field_bytes((int)f);
    return b < 0 ? 0 : b;
}

int sph_get(sph_engine *e, sph_field f, void *dst, size_t bytes)
{
    return e ? e->e->get((int)f, dst, bytes) : SPH_ERR_ARG;
}

int sph_set(sph_engine *e, sph_field f, const void *src, size_t bytes)
{
    return e ? e->e->set((int)f, src, bytes) : SPH_ERR_ARG;
}

int sph_write_bin(sph_engine *e, const char *path)
{
    return (e && path) ? e->e->write_bin(path) : SPH_ERR_ARG;
}

int sph_get_info(sph_engine *e, sph_info *info)
{
    if (!e || !info) return SPH_ERR_ARG;
    Engine &g = *e->e;
    int rc = g.poll_errors("info");
    std::memset(info, 0, sizeof *info);
    info->np = g.hs.np;
    info->nw = g.hs.nw;
    info->nb0 = g.hs.nb0;
    info->capacity = g.capacity;
    for (int d = 0; d < 3; ++d) info->num[d] = g.hs.num[d];
    info->periodic = g.hs.periodic;
    info->contactmodel = (int32_t)g.hs.contactmodel;
    info->precision = g.precision;
    info->fluid = g.hs.fluid;
    info->iter = g.last_ctl.iter;
    info->time = g.last_ctl.t_current;
    info->time_total = g.hs.t_total;
    info->dt = g.hs.dt;
    info->file_dt = g.hs.file_dt;
    info->step_count = g.hs.step_count;
    info->resorts = g.last_ctl.resorts;
    g.persist_describe(info);
    return rc;
}

int sph_time_sort(sph_engine *e, int reps, double *ms_per_sort)
{
    if (!e || !ms_per_sort || reps < 1) return SPH_ERR_ARG;
    Engine &g = *e->e;
    int rc = g.poll_errors("sort timing");
    if (rc < 0) return rc;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, g.stream);
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < reps && err == cudaSuccess; ++i) {
        err = sphb::launch_hash(g.P, g.S, g.stream);
        if (err == cudaSuccess) err = sphb::launch_resort(g.P, g.S, g.S.perm_scratch, 1, g.stream);
    }
    cudaEventRecord(b, g.stream);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (err != cudaSuccess) return g.cuda_fail(err, "sort timing");
    *ms_per_sort = ms / reps;
    return g.poll_errors("sort timing");
}

int sph_energy(sph_engine *e, const char *method, double *out)
{
    return e ? e->e->energy(method, out) : SPH_ERR_ARG;
}

int sph_porosity(sph_engine *e, int z_slices, double *z_pos, double *porosity)
{
    return e ? e->e->porosity_profile(z_slices, z_pos, porosity) : SPH_ERR_ARG;
}

int sph_render(sph_engine *e, int method, float max_val, float lower_cutoff, uint32_t width,
               uint32_t height, unsigned char *rgba)
{
    return e ? e->e->render(method, max_val, lower_cutoff, width, height, rgba) : SPH_ERR_ARG;
}

int sph_overlaps(sph_engine *e, uint32_t *pairs, double *delta, uint64_t capacity, uint64_t *count)
{
    return e ? e->e->overlaps(pairs, delta, capacity, count) : SPH_ERR_ARG;
}

const char *sph_last_error(sph_engine *e) { return e ? e->e->err.c_str() : "no engine"; }

void sph_close(sph_engine *e) { delete e; }

const char *sph_version(void)
{
    return "sphere_b200 0.1 (sm_100a; FP64 step kernels built with -fmad=false)";
}

}  // extern "C"
