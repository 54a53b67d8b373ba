// Engine object behind the C ABI.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "dem_state.h"
#include "host_state.h"
#include "../../include/sphere_b200.h"

namespace sphb {

struct DarcyDev;   // Darcy solver state (darcy.cu)
struct NSDev;      // Navier-Stokes solver state (navierstokes.cu)
struct MixedDev;   // mixed-precision state (dem_mixed.cu)
struct PersistDev; // fused persistent step path (engine_persist.cu)

// FP32 velocity copies of the mixed mode from the FP64 velocities.
cudaError_t launch_refresh_f(const DevParams &P, const DevState &S, cudaStream_t st);

class Engine {
public:
    ~Engine();

    // options
    int precision = 0;
    int integrator = 3;
    uint32_t capacity = 32;
    uint32_t nlmax = 48;          // neighbour-list entries per particle
    int verbose = 0;
    int graph_steps = 64;
    int warm_start = 0;
    int warm_start_train = 2000;  // solves the warm-start network trains on
    int step_kernel = 0;          // 0 automatic, 1 per-stage kernels, 2 persistent,
                                  // 3 per-stage with staged contacts, 4 per-stage with
                                  // contacts and integration in one launch
    uint32_t inject = 0;          // SPH_INJECT_* mask (a test knob; 0 in normal use)
    std::string outdir = "output";
    std::string sid = "unnamed";

    HostState hs;
    DevParams P{};
    DevState S{};
    cudaStream_t stream = nullptr;
    std::vector<void *> allocations;
    bool alloc_failed = false;    // a dalloc() returned null
    void *host_pinned = nullptr;
    unsigned char *tmp = nullptr;
    double4 *bond_f = nullptr, *bond_t = nullptr;

    // loop state mirrored on the host (same double additions as the device)
    double host_t = 0.0;
    int64_t host_iter = 0;
    double filetimeclock = 0.0;   // model time since the last file output
    DevCtl last_ctl{};

    cudaGraphExec_t graph_exec = nullptr;
    int graph_view = -1;          // state view the graph was captured with
    bool graph_fused = false;     // the graph holds fused per-stage steps
    bool graph_failed = false;
    bool warmed = false;

    std::string err;

    DarcyDev *darcy = nullptr;
    NSDev *ns = nullptr;
    MixedDev *mixed = nullptr;
    PersistDev *persist = nullptr;
    DevState S_view[2]{};         // S_view[v]: buffer view v (S is the current one)
    int cur_view = 0;
    bool persist_off = false;     // the autotuner found the per-stage kernels faster
    // per-stage steps with the contact search and the particle integration
    // in one launch (k_contacts_integrate into the other buffer of the
    // x / vel / angvel pair, then k_walls_step); each step flips the view
    bool fused = false;
    int view_upload = 0;          // host source of the view copied to the persistent kernel
    FILE *convlog = nullptr;
    int jacobi_grid = 0;            // blocks of the cooperative Jacobi launch
    int darcy_exact_stop = 0;       // 1: stop at the first converged iteration
    bool darcy_keep_dphi = false;   // this step ends at a file output
    unsigned darcy_wall0_iz = 10000000u;

    int fail(int code, const std::string &msg);
    int cuda_fail(cudaError_t e, const char *where);
    template <class T> T *dalloc(size_t n);

    void build_params();
    int allocate_and_upload();
    int poll_errors(const char *where);
    cudaError_t enqueue_stage(int stage);
    cudaError_t enqueue_step();
    cudaError_t enqueue_fluid();
    int profile(uint64_t n, struct sph_profile *out);
    int ensure_graph();
    cudaGraphExec_t capture_steps(int k);
    cudaError_t launch_trial_steps(cudaGraphExec_t g, uint64_t n);
    int stages_after(uint64_t n);
    int step(uint64_t n);
    int step_stages(uint64_t n);
    void advance_host_clock(uint64_t n);
    int64_t field_bytes(int f) const;
    double4 *sorted_vec(int f) const;
    double *sorted_scalar(int f) const;
    int get(int f, void *dst, size_t bytes);
    int get_distmod(double *dst);
    int get_delta_t_mixed(double *dst);
    int set(int f, const void *src, size_t bytes);
    int download_state();
    int write_bin(const char *path);
    int write_status();
    int run();

    // Darcy (cfd_solver 1); no-ops for dry runs
    int darcy_init();
    int darcy_sync_wall();
    void darcy_set_host_wall();
    void darcy_free();
    int64_t darcy_field_bytes(int f) const;
    int darcy_get(int f, void *dst, size_t bytes);
    int darcy_download();
    int step_with_fluid_log(uint64_t n);
    // Navier-Stokes (cfd_solver 0, navierstokes.cu)
    int ns_init();
    void ns_free();
    void ns_set_host_wall();
    cudaError_t enqueue_ns();
    int64_t ns_field_bytes(int f) const;
    int ns_get(int f, void *dst, size_t bytes);
    int ns_download();
    int ns_check_stability();
    int ns_step_with_log(uint64_t n);
    void conv_open();
    void conv_close();

    // diagnostics on the resident state (stats.cu)
    int energy(const char *method, double *out);
    int porosity_profile(int z_slices, double *z_pos, double *porosity);
    int overlaps(uint32_t *pairs, double *delta, uint64_t cap, uint64_t *count);
    int render(int method, float max_val, float lower_cutoff, unsigned width, unsigned height,
               unsigned char *rgba);

    // mixed precision
    int mixed_init();

    // fused per-stage step path
    bool fused_eligible() const;
    void set_fused(bool on);
    void flip_view();
    int graph_len() const;

    // fused persistent step path
    bool persist_eligible() const;
    void make_views();
    int persist_init();
    void persist_free();
    unsigned persist_grid(int shape) const;
    cudaError_t persist_launch(uint64_t n, int shape, unsigned grid);
    int step_persistent(uint64_t n);
    int persist_after(uint64_t n);
    void *persist_ctl() const;    // the box's PersistCtl on the device
    void persist_describe(struct sph_info *info) const;
};

// Opens one engine from a .bin path (path != null) or from its bytes.
int open_engine(const char *path, const void *bytes, size_t nbytes, const struct sph_opts *opts,
                const char *sid, std::unique_ptr<Engine> &out, std::string &err);

// Zero-filled device array owned by the engine (released in ~Engine).
template <class T> T *Engine::dalloc(size_t n)
{
    void *p = nullptr;
    size_t bytes = n ? n * sizeof(T) : sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        alloc_failed = true;
        return nullptr;
    }
    cudaMemsetAsync(p, 0, bytes, stream);
    allocations.push_back(p);
    return (T *)p;
}

}  // namespace sphb
