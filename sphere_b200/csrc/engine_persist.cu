// The engine's fused persistent step path (persistent.cuh) for one box:
// state views for the ping-pong buffers, the launch, and an autotuner that
// picks the block shape and grid from timed trial launches made of real
// steps (every shape computes the same results, so trials change nothing
// but the clock).
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine_internal.h"
#include "persistent_launch.h"
#include "dem_launch.h"

namespace sphb {

struct PersistDev {
    PersistCtl *pc = nullptr;
    BoxRec *table = nullptr;
    unsigned *order = nullptr;
    unsigned char *sync = nullptr;    // next counter, abort flag, group barriers
    size_t sync_bytes = 0;
    int shape = 1;
    unsigned grid = 0;
    bool tuned = false;
    int sms = 0;
};

namespace {

__global__ void k_refresh_f(DevParams P, DevState S)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.np || !S.vel_f) return;
    double4 v = S.vel[k], w = S.angvel[k];
    S.vel_f[k] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
    S.angvel_f[k] = make_float4((float)w.x, (float)w.y, (float)w.z, 0.0f);
}

}  // namespace

cudaError_t launch_refresh_f(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0 || !S.vel_f) return cudaSuccess;
    k_refresh_f<<<(P.np + 255) / 256, 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

// Both fused step paths integrate inside the contact pass, so they cover
// dry runs without bonds or the shear-stress wall: those forces would have
// to join the contact forces before the integration.
bool Engine::fused_eligible() const
{
    return !hs.fluid && hs.nb0 == 0 && !(hs.nw > 0 && hs.wmode[0] == 3) && hs.np > 0;
}

bool Engine::persist_eligible() const
{
    if (step_kernel != 0 && step_kernel != 2) return false;
    return fused_eligible();
}

// Selects the per-stage step kernels: the contact and integration kernels
// (on == false) or k_contacts_integrate + k_walls_step.  A graph of the
// other kind is dropped, and the next step runs eagerly first (kernel
// attributes are set outside any capture).
void Engine::set_fused(bool on)
{
    if (on == fused) return;
    fused = on;
    warmed = false;
    if (graph_exec) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
}

void Engine::flip_view()
{
    cur_view ^= 1;
    S = S_view[cur_view];
}

// Steps per captured graph: even on the fused per-stage path, so every
// replay starts and ends on the view the graph was captured with.
int Engine::graph_len() const
{
    return graph_steps + ((fused && (graph_steps & 1)) ? 1 : 0);
}

void Engine::make_views()
{
    S_view[0] = S;
    S_view[1] = S;
    std::swap(S_view[1].x, S_view[1].x_nx);
    std::swap(S_view[1].vel, S_view[1].vel_nx);
    std::swap(S_view[1].angvel, S_view[1].angvel_nx);
    std::swap(S_view[1].vel_f, S_view[1].vel_f_nx);
    std::swap(S_view[1].angvel_f, S_view[1].angvel_f_nx);
}

int Engine::persist_init()
{
    if (!persist_eligible()) return ST_OK;
    persist = new PersistDev();
    PersistDev &D = *persist;
    D.pc = dalloc<PersistCtl>(1);
    D.table = dalloc<BoxRec>(1);
    D.order = dalloc<unsigned>(1);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&D.sms, cudaDevAttrMultiProcessorCount, dev);
    // one group: the whole grid steps the box
    D.sync_bytes = sync_bytes(1);
    D.sync = dalloc<unsigned char>(D.sync_bytes);
    if (!D.pc || !D.table || !D.order || !D.sync) return fail(ST_CUDA, "device allocation failed");
    BoxRec r;
    std::memset(&r, 0, sizeof r);
    r.P = P;
    r.S[0] = S_view[0];
    r.S[1] = S_view[1];
    r.pc = D.pc;
    r.scratch = S.perm_scratch;
    r.nblk = P.nblocks256;
    unsigned zero = 0;
    cudaMemcpyAsync(D.table, &r, sizeof r, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(D.order, &zero, 4, cudaMemcpyHostToDevice, stream);
    cudaError_t e = launch_refresh_f(P, S, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "persistent setup");
    D.shape = 1;
    D.grid = persist_grid(D.shape);
    if (D.grid == 0) return fail(ST_CUDA, "persistent step kernel cannot be resident");
    return ST_OK;
}

void *Engine::persist_ctl() const { return persist ? (void *)persist->pc : nullptr; }

void Engine::persist_describe(sph_info *info) const
{
    info->step_path = (persist && !persist_off) ? 1 : (fused ? 2 : 0);
    info->step_threads = persist ? kPersistShapes[persist->shape].threads : 0;
    info->step_grid = persist ? (int32_t)persist->grid : 0;
    info->tuned = persist ? (persist->tuned ? 1 : 0) : 0;
}

void Engine::persist_free()
{
    delete persist;
    persist = nullptr;
}

unsigned Engine::persist_grid(int shape) const
{
    const int prec = precision;
    const int threads = kPersistShapes[shape].threads;
    size_t smem = persistent_smem(threads, capacity);
    int per_sm = persistent_blocks_per_sm(prec, (int)hs.contactmodel, shape, smem);
    if (per_sm <= 0) return 0;
    unsigned grid = (unsigned)(per_sm * persist->sms);
    unsigned need = (unsigned)((hs.np + threads - 1) / threads);
    return std::max(1u, std::min(grid, need));
}

cudaError_t Engine::persist_launch(uint64_t n, int shape, unsigned grid)
{
    PersistDev &D = *persist;
    const int threads = kPersistShapes[shape].threads;
    cudaError_t e = cudaMemsetAsync(D.sync, 0, D.sync_bytes, stream);
    if (e != cudaSuccess) return e;
    // the per-stage fused steps flip the view on the host
    view_upload = cur_view;
    e = cudaMemcpyAsync(&D.pc->view, &view_upload, sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    BatchArgs A;
    A.boxes = D.table;
    A.nbox = 1;
    A.order = D.order;
    set_sync_args(A, D.sync);
    A.group_size = grid;
    A.nsteps = (unsigned)n;
    A.inject = (inject & kInjectPersistent) ? 1u : 0u;
    return persistent_launch(precision, (int)hs.contactmodel, shape, A, grid,
                             persistent_smem(threads, capacity), stream);
}

// Runs n steps on the persistent path.  The first call with enough steps
// times each block shape -- and, unless the persistent path was requested
// explicitly, the per-stage kernels -- on real steps and keeps the fastest.
int Engine::step_persistent(uint64_t n)
{
    PersistDev &D = *persist;
    uint64_t done = 0;
    const uint64_t trial = 8;
    // candidates: every block shape of the persistent kernel, then (unless
    // the persistent path was requested) the per-stage kernels and the
    // per-stage kernels with contacts and integration in one launch
    const int ncand = kNumPersistShapes + (step_kernel == 2 ? 0 : 2);
    if (!D.tuned && n >= trial * (uint64_t)(ncand + 2)) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        float best = 1e30f;
        int best_cand = D.shape;
        int rc = ST_OK;
        cudaGraphExec_t trial_graph = nullptr;
        for (int cand = 0; cand < ncand && rc == ST_OK; ++cand) {
            const bool stages = cand >= kNumPersistShapes;
            unsigned g = stages ? 1 : persist_grid(cand);
            if (!g) continue;
            if (stages) {
                set_fused(cand == kNumPersistShapes + 1);
                if (trial_graph) {
                    cudaGraphExecDestroy(trial_graph);
                    trial_graph = nullptr;
                }
                // warm the per-stage path: the eager first step, then the
                // trial steps as one graph (as they run in production; eager
                // launches would time the host, not the kernels)
                rc = step_stages(1);
                done += 1;
                if (rc) break;
                trial_graph = capture_steps((int)trial);
                cudaError_t e = launch_trial_steps(trial_graph, trial);
                if (e != cudaSuccess) rc = cuda_fail(e, "step");
                done += trial;
                if (rc || (rc = stages_after(trial))) break;
            }
            cudaEventRecord(a, stream);
            cudaError_t e = stages ? launch_trial_steps(trial_graph, trial) : persist_launch(trial, cand, g);
            cudaEventRecord(b, stream);
            if (e != cudaSuccess) rc = cuda_fail(e, stages ? "step" : "persistent step");
            if (rc) break;
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            done += trial;
            if ((rc = stages ? stages_after(trial) : persist_after(trial))) break;
            if (ms < best) {
                best = ms;
                best_cand = cand;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (trial_graph) cudaGraphExecDestroy(trial_graph);
        if (rc) return rc;
        D.tuned = true;
        if (best_cand >= kNumPersistShapes) {
            persist_off = true;
            set_fused(best_cand == kNumPersistShapes + 1);
            return step_stages(n - done);
        }
        set_fused(false);
        D.shape = best_cand;
        D.grid = persist_grid(best_cand);
    }
    if (done < n) {
        cudaError_t e = persist_launch(n - done, D.shape, D.grid);
        if (e != cudaSuccess) return cuda_fail(e, "persistent step");
        return persist_after(n - done);
    }
    return ST_OK;
}

// Enqueues the n per-stage steps of a tuning trial: one replay of the
// n-step graph, or eager launches when it could not be captured.  Nothing
// waits on the host, so the events around it time the device alone.
cudaError_t Engine::launch_trial_steps(cudaGraphExec_t g, uint64_t n)
{
    if (g) return cudaGraphLaunch(g, stream);
    cudaError_t e = cudaSuccess;
    for (uint64_t i = 0; i < n && e == cudaSuccess; ++i) e = enqueue_step();
    return e;
}

// After n per-stage trial steps: the host clock and device errors.
int Engine::stages_after(uint64_t n)
{
    advance_host_clock(n);
    return poll_errors("step");
}

// After a launch of n steps: advance the host mirrors, pick up the current
// view and report device errors.
int Engine::persist_after(uint64_t n)
{
    PersistDev &D = *persist;
    int view = 0, abort = 0;
    cudaMemcpyAsync(&view, &D.pc->view, 4, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&abort, D.sync + 4, 4, cudaMemcpyDeviceToHost, stream);
    advance_host_clock(n);
    int rc = poll_errors("step");
    cur_view = view & 1;
    S = S_view[cur_view];
    if (rc) return rc;
    if (abort) return fail(ST_TIMEOUT, "step: a bounded device wait timed out");
    return ST_OK;
}

}  // namespace sphb
