// Batch engine: many independent boxes (uneven particle counts) stepped by
// one launch of the persistent step kernel.
//
// Each box is a full engine (its own state, parameters, walls and clock);
// the batch owns a table of the boxes' state views and launches the fused
// step kernel over all of them.  Groups of `group_size` blocks take boxes
// from a work counter, largest first, and run all requested steps of a box
// before taking the next, so a box's working set stays in L2 while it is
// stepped and no grid-wide barrier is needed.  The block shape and group
// size come from a project-written autotuner that times short trial
// launches made of real steps (all configurations compute identical
// results).  Repeated step calls of the same length replay a CUDA graph of
// the launch.
#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "persistent_launch.h"
#include "../../include/sphere_b200.h"

namespace sphb {

struct BatchEngine {
    std::vector<std::unique_ptr<Engine>> boxes;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    BoxRec *table = nullptr;
    unsigned *order = nullptr;
    unsigned char *sync = nullptr;
    size_t sync_bytes = 0;
    int prec = 0, model = 2;
    unsigned ncmax = 1;
    int sms = 0;
    // launch configuration
    int shape = 1;
    unsigned gsz = 1, grid = 0;
    bool tuned = false;
    std::vector<sph_batch_trial> trials;
    // graph of one launch of graph_n steps
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_n = 0;
    bool graph_failed = false;
    std::string err;

    ~BatchEngine()
    {
        if (graph) cudaGraphExecDestroy(graph);
        for (void *p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    int fail(int code, const std::string &m)
    {
        err = m;
        return code;
    }
    int cuda_fail(cudaError_t e, const char *where)
    {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return ST_CUDA;
    }
    template <class T> T *alloc(size_t n)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
        allocs.push_back(p);
        return (T *)p;
    }

    unsigned grid_for(int sh, unsigned g) const
    {
        const int threads = kPersistShapes[sh].threads;
        int per_sm = persistent_blocks_per_sm(prec, model, sh, persistent_smem(threads, ncmax));
        if (per_sm <= 0) return 0;
        unsigned resident = (unsigned)(per_sm * sms);
        if (g > resident) return 0;
        // no more groups than boxes, and every group of g blocks
        unsigned groups = std::min<unsigned>(resident / g, (unsigned)boxes.size());
        return groups * g;
    }

    cudaError_t enqueue(uint64_t n, int sh, unsigned g, unsigned gr)
    {
        cudaError_t e = cudaMemsetAsync(sync, 0, sphb::sync_bytes(gr / g), stream);
        if (e != cudaSuccess) return e;
        BatchArgs A;
        A.boxes = table;
        A.nbox = (unsigned)boxes.size();
        A.order = order;
        set_sync_args(A, sync);
        A.group_size = g;
        A.nsteps = (unsigned)n;
        A.inject = (boxes[0]->inject & sphb::kInjectPersistent) ? 1u : 0u;
        return persistent_launch(prec, model, sh, A, gr,
                                 persistent_smem(kPersistShapes[sh].threads, ncmax), stream);
    }

    // After n steps: the boxes' host mirrors, and errors.
    int after(uint64_t n)
    {
        int flags[2] = {0, 0};
        cudaError_t e = cudaMemcpyAsync(flags, sync + 4, 8, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "batch step");
        for (auto &b : boxes) {
            b->advance_host_clock(n);
            b->cur_view ^= (int)(n & 1);
            b->S = b->S_view[b->cur_view];
        }
        if (flags[0] || flags[1]) {
            // find the box that failed and its message
            for (size_t i = 0; i < boxes.size(); ++i) {
                Engine &b = *boxes[i];
                int v = 0;
                cudaMemcpy(&v, &reinterpret_cast<PersistCtl *>(b.persist_ctl())->view, 4,
                           cudaMemcpyDeviceToHost);
                b.cur_view = v & 1;
                b.S = b.S_view[b.cur_view];
                int rc = b.poll_errors("batch step");
                if (rc) return fail(rc, "box " + std::to_string(i) + ": " + b.err);
            }
            if (flags[0]) return fail(ST_TIMEOUT, "batch step: a bounded device wait timed out");
        }
        return ST_OK;
    }

    int launch(uint64_t n, int sh, unsigned g, unsigned gr)
    {
        cudaError_t e = enqueue(n, sh, g, gr);
        if (e != cudaSuccess) return cuda_fail(e, "batch step");
        return after(n);
    }

    // Times every (block shape, group size) on `trial` real steps each and
    // keeps the fastest.
    int autotune(uint64_t trial, uint64_t &done)
    {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        float best = 1e30f;
        int rc = ST_OK;
        for (int sh = 0; sh < kNumPersistShapes && rc == ST_OK; ++sh)
            for (unsigned g = 1; g <= 64 && rc == ST_OK; g *= 2) {
                unsigned gr = grid_for(sh, g);
                if (!gr) continue;
                cudaEventRecord(a, stream);
                cudaError_t e = enqueue(trial, sh, g, gr);
                cudaEventRecord(b, stream);
                if (e != cudaSuccess) {
                    rc = cuda_fail(e, "batch autotune");
                    break;
                }
                cudaEventSynchronize(b);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, a, b);
                rc = after(trial);
                done += trial;
                sph_batch_trial t;
                t.threads = kPersistShapes[sh].threads;
                t.group_size = (int)g;
                t.grid = (int)gr;
                t.ms_per_step = ms / (double)trial;
                trials.push_back(t);
                if (ms < best) {
                    best = ms;
                    shape = sh;
                    gsz = g;
                    grid = gr;
                }
            }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        tuned = true;
        return rc;
    }

    int step(uint64_t n, bool allow_tune)
    {
        if (n == 0) return ST_OK;
        uint64_t done = 0;
        const uint64_t trial = 4;
        if (!tuned && allow_tune && n >= trial * 64) {
            int rc = autotune(trial, done);
            if (rc) return rc;
        }
        uint64_t left = n - done;
        if (left == 0) return ST_OK;
        // a captured launch of `left` steps is replayed by later calls of the
        // same length
        if (!graph_failed && (graph == nullptr || graph_n != left)) {
            if (graph) {
                cudaGraphExecDestroy(graph);
                graph = nullptr;
            }
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t e1 = enqueue(left, shape, gsz, grid);
                cudaError_t e2 = cudaStreamEndCapture(stream, &g);
                if (e1 == cudaSuccess && e2 == cudaSuccess && g &&
                    cudaGraphInstantiate(&graph, g, 0) == cudaSuccess)
                    graph_n = left;
                else
                    graph = nullptr;
                if (g) cudaGraphDestroy(g);
            }
            if (!graph) {
                graph_failed = true;
                cudaGetLastError();
            }
        }
        if (graph) {
            cudaError_t e = cudaGraphLaunch(graph, stream);
            if (e != cudaSuccess) return cuda_fail(e, "batch graph launch");
            return after(left);
        }
        return launch(left, shape, gsz, grid);
    }
};

}  // namespace sphb

using sphb::BatchEngine;

struct sph_batch {
    std::unique_ptr<BatchEngine> b;
};

namespace {
thread_local std::string g_batch_open_error;

int batch_open(int nbox, const char *const *paths, const void *const *bufs, const size_t *sizes,
               const sph_opts *opts, sph_batch **out)
{
    if (!out || nbox <= 0) return SPH_ERR_ARG;
    *out = nullptr;
    auto B = std::make_unique<BatchEngine>();
    if (opts && opts->struct_size != sizeof(sph_opts)) {
        g_batch_open_error = "sph_opts.struct_size does not match this library's sph_opts";
        return SPH_ERR_ARG;
    }
    sph_opts o;
    if (opts) {
        o = *opts;
    } else {
        o.struct_size = sizeof(sph_opts);
        sph_default_opts(&o);
    }
    o.step_kernel = 2;   // every box must run on the fused step
    o.fluid = 0;
    for (int i = 0; i < nbox; ++i) {
        std::unique_ptr<sphb::Engine> e;
        std::string err;
        std::string sid = "box" + std::to_string(i);
        int rc = sphb::open_engine(paths ? paths[i] : nullptr, bufs ? bufs[i] : nullptr,
                                   sizes ? sizes[i] : 0, &o, sid.c_str(), e, err);
        if (rc < 0) {
            g_batch_open_error = "box " + std::to_string(i) + ": " + err;
            return rc;
        }
        B->boxes.push_back(std::move(e));
    }
    B->prec = o.precision;
    B->model = (int)B->boxes[0]->hs.contactmodel;
    for (auto &e : B->boxes) {
        if ((int)e->hs.contactmodel != B->model) {
            g_batch_open_error = "all boxes of a batch must use the same contact model";
            return SPH_ERR_UNSUPPORTED;
        }
        B->ncmax = std::max(B->ncmax, e->capacity);
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) {
        g_batch_open_error = "cudaStreamCreate failed";
        return SPH_ERR_CUDA;
    }
    const size_t nb = B->boxes.size();
    B->table = B->alloc<sphb::BoxRec>(nb);
    B->order = B->alloc<unsigned>(nb);
    B->sync_bytes = sphb::sync_bytes((unsigned)B->sms * 32);
    B->sync = B->alloc<unsigned char>(B->sync_bytes);
    if (!B->table || !B->order || !B->sync) {
        g_batch_open_error = "device allocation failed";
        return SPH_ERR_CUDA;
    }
    std::vector<sphb::BoxRec> recs(nb);
    for (size_t i = 0; i < nb; ++i) {
        sphb::Engine &e = *B->boxes[i];
        cudaStreamSynchronize(e.stream);
        sphb::BoxRec &r = recs[i];
        std::memset(&r, 0, sizeof r);
        r.P = e.P;
        r.S[0] = e.S_view[0];
        r.S[1] = e.S_view[1];
        r.pc = reinterpret_cast<sphb::PersistCtl *>(e.persist_ctl());
        r.scratch = e.S.perm_scratch;
        r.nblk = e.P.nblocks256;
    }
    std::vector<unsigned> ord(nb);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](unsigned a, unsigned b) {
        return B->boxes[a]->hs.np > B->boxes[b]->hs.np;
    });
    cudaMemcpy(B->table, recs.data(), nb * sizeof(sphb::BoxRec), cudaMemcpyHostToDevice);
    cudaMemcpy(B->order, ord.data(), nb * 4, cudaMemcpyHostToDevice);
    // default before tuning: one block of 128 threads per box
    B->shape = 1;
    B->gsz = 1;
    B->grid = B->grid_for(1, 1);
    if (!B->grid) {
        g_batch_open_error = "persistent step kernel cannot be resident";
        return SPH_ERR_CUDA;
    }
    *out = new sph_batch{std::move(B)};
    return SPH_OK;
}
}  // namespace

extern "C" {

int sph_open_batch(const char *const *bin_paths, int nbox, const sph_opts *opts, sph_batch **out)
{
    if (!bin_paths) return SPH_ERR_ARG;
    return batch_open(nbox, bin_paths, nullptr, nullptr, opts, out);
}

int sph_open_batch_buffers(const void *const *bufs, const size_t *sizes, int nbox,
                           const sph_opts *opts, sph_batch **out)
{
    if (!bufs || !sizes) return SPH_ERR_ARG;
    return batch_open(nbox, nullptr, bufs, sizes, opts, out);
}

const char *sph_batch_open_error(void) { return g_batch_open_error.c_str(); }

int sph_batch_step(sph_batch *b, uint64_t n) { return b ? b->b->step(n, true) : SPH_ERR_ARG; }

int sph_batch_step_timed(sph_batch *b, uint64_t n, double *device_ms)
{
    if (!b || !device_ms) return SPH_ERR_ARG;
    BatchEngine &B = *b->b;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, B.stream);
    int rc = B.step(n, false);
    cudaEventRecord(e1, B.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *device_ms = ms;
    return rc;
}

int sph_batch_autotune(sph_batch *b, uint64_t trial_steps)
{
    if (!b) return SPH_ERR_ARG;
    uint64_t done = 0;
    return b->b->autotune(trial_steps ? trial_steps : 4, done);
}

int sph_batch_size(sph_batch *b) { return b ? (int)b->b->boxes.size() : SPH_ERR_ARG; }

int64_t sph_batch_field_bytes(sph_batch *b, int box, sph_field f)
{
    if (!b || box < 0 || box >= (int)b->b->boxes.size()) return SPH_ERR_ARG;
    int64_t n = b->b->boxes[box]->field_bytes((int)f);
    return n < 0 ? 0 : n;
}

int sph_batch_get(sph_batch *b, int box, sph_field f, void *dst, size_t bytes)
{
    if (!b || box < 0 || box >= (int)b->b->boxes.size()) return SPH_ERR_ARG;
    BatchEngine &B = *b->b;
    cudaStreamSynchronize(B.stream);
    sphb::Engine &e = *B.boxes[box];
    int rc = e.get((int)f, dst, bytes);
    if (rc < 0) B.err = e.err;
    return rc;
}

int sph_batch_write_bin(sph_batch *b, int box, const char *path)
{
    if (!b || !path || box < 0 || box >= (int)b->b->boxes.size()) return SPH_ERR_ARG;
    BatchEngine &B = *b->b;
    cudaStreamSynchronize(B.stream);
    int rc = B.boxes[box]->write_bin(path);
    if (rc < 0) B.err = B.boxes[box]->err;
    return rc;
}

int sph_batch_get_config(sph_batch *b, sph_batch_config *cfg)
{
    if (!b || !cfg) return SPH_ERR_ARG;
    BatchEngine &B = *b->b;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->threads = sphb::kPersistShapes[B.shape].threads;
    cfg->group_size = (int)B.gsz;
    cfg->grid = (int)B.grid;
    cfg->tuned = B.tuned ? 1 : 0;
    cfg->ntrials = (int)B.trials.size();
    cfg->graph = B.graph ? 1 : 0;
    return SPH_OK;
}

int sph_batch_get_trials(sph_batch *b, sph_batch_trial *out, int max)
{
    if (!b || (!out && max > 0)) return SPH_ERR_ARG;
    int n = std::min<int>(max, (int)b->b->trials.size());
    for (int i = 0; i < n; ++i) out[i] = b->b->trials[i];
    return (int)b->b->trials.size();
}

const char *sph_batch_last_error(sph_batch *b) { return b ? b->b->err.c_str() : "no batch"; }

void sph_batch_close(sph_batch *b) { delete b; }

}  // extern "C"
