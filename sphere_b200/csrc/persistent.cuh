// Persistent DEM step kernel: many DEM steps of one or many boxes in one
// launch.
//
// The grid is split into groups of `group_size` blocks.  A group takes the
// next box from a work counter (boxes listed largest first) and runs all
// `nsteps` steps of it before taking another.  Per step:
//
//   [re-sort, when the previous step moved a particle to another cell]
//   C: per particle (group-stride): neighbour-list rebuild when needed,
//      contact search + forces, integration into the other buffer of the
//      x/vel/angvel ping-pong pair;
//   -- group barrier --
//   W: wall-force partial sums (the reference's 256-particle trees over
//      original indices); the block that finishes last adds them in order,
//      moves the walls, advances the clock and publishes the next step's
//      flags;
//   -- group barrier --
//
// Integration reads only the particle's own state and the forces this
// thread just computed, while the contact search of other particles reads
// the untouched current buffer, so fusing the two stages needs no barrier
// between them.  The arithmetic is the per-stage kernels' (same device
// functions, same operation order), so faithful and FP64 modes stay
// bit-identical to the oracle.  A group of one block synchronises with
// __syncthreads only; larger groups use a bounded software barrier, which
// needs every block resident: the kernel is always launched cooperatively.
#pragma once

#include "dem_device.cuh"
#include "reduce_device.cuh"
#include "resort_device.cuh"

namespace sphb {

// Loop state a step starts from, published by the previous step's finalizer.
struct StepHead {
    long long iter;
    double t_current;
    int velocity_state;
    int err;
    int resort, nl;       // raised by the previous step
    int view;             // index of the current buffer view
    int pad;
};

// Per-box control block of the persistent path.
struct PersistCtl {
    StepHead head[2];          // indexed by the parity of `iter`
    int flag_resort[2];        // raised during the step of that parity
    int flag_nl[2];
    unsigned ticket;           // blocks done with the W phase
    int view;                  // current view between launches
};

// One box: its parameters and two views of its state that differ only in
// which buffer of each ping-pong pair is current (S[v].x is current,
// S[v].x_nx the other).
struct BoxRec {
    DevParams P;
    DevState S[2];
    PersistCtl *pc;
    unsigned char *scratch;    // re-sort scratch (make_perm_scratch)
    unsigned nblk;             // ceil(np / 256): the reference's block count
    unsigned pad;
};

// Barrier state of one group: the arrival counter and the generation the
// waiters poll sit on different 128-byte lines.  Groups of more than 64
// blocks arrive through 16 sub-counters first (sub[], one line each).
struct GroupSync {
    unsigned count;
    int box;
    unsigned pad0[30];
    unsigned gen;
    unsigned pad1[31];
};
constexpr int kBarrierSubs = 16;
struct GroupTree {
    unsigned sub[kBarrierSubs][32];
};

struct BatchArgs {
    const BoxRec *boxes;
    unsigned nbox;
    const unsigned *order;     // processing order (largest box first)
    unsigned *next;            // work counter, zero at launch
    GroupSync *groups;         // zero at launch
    GroupTree *tree;           // zero at launch; sub-counters of group 0
    unsigned group_size;
    unsigned nsteps;
    int *abort;                // set when a barrier gave up; every group stops
    int *any_err;              // set when some box raised an error
    unsigned inject;           // 1: the group barriers never release (a test knob)
};

// Barrier over the blocks of one group, bounded: after ~2^24 polls it sets
// *abort and returns false, and every waiting block returns false as soon
// as it sees *abort.  Groups of more than 64 blocks (only ever group 0: a
// single box stepped by the whole grid) arrive in two levels so no counter
// takes more than ~64 serialised atomics.  With `inject` no block releases
// the barrier and every block gives up after kInjectPolls polls.
__device__ __forceinline__ bool group_barrier(GroupSync *g, GroupTree *tree, unsigned size,
                                              unsigned rank, int *abort, bool inject)
{
    if (size == 1) {
        __syncthreads();
        if (inject && threadIdx.x == 0) atomicExch(abort, 1);
        return !inject;
    }
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &g->gen;
        const unsigned cur = *gen;
        __threadfence();
        bool last;
        if (size > 64) {
            const unsigned s = rank % kBarrierSubs;
            const unsigned members = (size - s + kBarrierSubs - 1) / kBarrierSubs;
            last = false;
            if (atomicAdd(&tree->sub[s][0], 1u) == members - 1) {
                tree->sub[s][0] = 0;
                __threadfence();
                last = atomicAdd(&g->count, 1u) == kBarrierSubs - 1;
            }
        } else {
            last = atomicAdd(&g->count, 1u) == size - 1;
        }
        ok = 1;
        if (last && !inject) {
            g->count = 0;
            __threadfence();
            atomicAdd(&g->gen, 1u);
        } else {
            unsigned spins = 0, nap = 32;
            const unsigned limit = inject ? kInjectPolls : (1u << 24);
            while (inject || *gen == cur) {
                if (++spins > limit) {
                    atomicExch(abort, 1);
                    ok = 0;
                    break;
                }
                if (*(volatile int *)abort) {
                    ok = 0;
                    break;
                }
                __nanosleep(nap);
                if (nap < 256) nap <<= 1;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Dynamic shared memory: the slot rows (NT * nc u32, at least 16 KB so the
// same space stages the ordered wall-force sum).  NT threads per block,
// MINB resident blocks per SM (register budget 65536 / (NT * MINB)).
template <int PREC, int MODEL, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_persistent(BatchArgs A)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    uint32_t *srow = reinterpret_cast<uint32_t *>(dyn);
    double *stage = reinterpret_cast<double *>(dyn);
    __shared__ BoxRec box;
    __shared__ double cache[256];
    __shared__ StepHead h;
    __shared__ int s_box;
    // this block's copy of the walls: every block moves them identically
    // from the same partial sums, block 0 of the group publishes them
    __shared__ double4 sw_nx[6], sw_mvfd[6];
    __shared__ double sw_acc[6];
    __shared__ double4 *g_wnx, *g_wmvfd;
    __shared__ double *g_wacc;

    const unsigned gsz = A.group_size;
    const unsigned gid = blockIdx.x / gsz, rank = blockIdx.x % gsz;
    GroupSync *G = &A.groups[gid];
    const unsigned B = blockDim.x, t = threadIdx.x;
    const unsigned gtid = rank * B + t, gstride = gsz * B;
    auto bar = [&]() { return group_barrier(G, A.tree, gsz, rank, A.abort, A.inject != 0); };

    for (;;) {
        // ---- take the next box ----
        if (rank == 0 && t == 0) {
            unsigned i = atomicAdd(A.next, 1u);
            G->box = i < A.nbox ? (int)A.order[i] : -1;
        }
        if (!bar()) return;
        if (t == 0) s_box = *(volatile int *)&G->box;
        __syncthreads();
        const int bi = s_box;
        if (bi < 0) return;
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&A.boxes[bi]);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&box);
            for (unsigned i = t; i < sizeof(BoxRec) / 4; i += B) dst[i] = src[i];
        }
        __syncthreads();
        if (t == 0) {
            // the loop state as the host (or the last launch) left it;
            // nothing writes it before this box's first W phase
            const DevCtl *ctl = box.S[0].ctl;
            h.iter = *(volatile long long *)&ctl->iter;
            h.t_current = *(volatile double *)&ctl->t_current;
            h.velocity_state = *(volatile int *)&ctl->velocity_state;
            h.err = *(volatile int *)&ctl->err;
            h.resort = *(volatile int *)&ctl->resort;
            h.nl = *(volatile int *)&ctl->nl_rebuild;
            h.view = *(volatile int *)&box.pc->view;
            g_wnx = box.S[0].wnx;
            g_wmvfd = box.S[0].wmvfd;
            g_wacc = box.S[0].wacc;
            for (unsigned w = 0; w < box.P.nw && w < 6; ++w) {
                sw_nx[w] = ldcg4(&g_wnx[w]);
                sw_mvfd[w] = ldcg4(&g_wmvfd[w]);
                sw_acc[w] = __ldcg(&g_wacc[w]);
            }
            for (int v = 0; v < 2; ++v) {
                box.S[v].wnx = sw_nx;
                box.S[v].wmvfd = sw_mvfd;
                box.S[v].wacc = sw_acc;
            }
            if (rank == 0) {
                // flags a previous launch left behind were carried into ctl
                PersistCtl *pc = box.pc;
                pc->flag_resort[0] = pc->flag_resort[1] = 0;
                pc->flag_nl[0] = pc->flag_nl[1] = 0;
            }
        }
        // every block has read the loop state before any block changes it
        if (!bar()) return;
        const DevParams &P = box.P;
        PersistCtl *pc = box.pc;

        for (unsigned s = 0; s < A.nsteps; ++s) {
            if (h.err) break;
            const int v = h.view;
            const DevState &S = box.S[v];
            const long long iter = h.iter;
            bool nl = h.nl != 0;
            const bool resorted = h.resort != 0;
            // ---- re-sort ----
            if (resorted) {
                PermScratch W = make_perm_scratch(box.scratch, P.np);
                if (!resort_group(P, S, W, gsz, rank, bar, PREC == 2)) {
                    if (t == 0) raise_err(S.ctl, DERR_TIMEOUT, -1);
                    return;
                }
                if (!bar()) return;
                nl = true;
            }
            // ---- C: contacts + integration ----
            StepClock clk;
            clk.iter = iter;
            clk.t_current = h.t_current;
            clk.velocity_state = h.velocity_state;
            clk.tau_eff_x = 0.0;
            int *fr = &pc->flag_resort[iter & 1], *fn = &pc->flag_nl[iter & 1];
            for (unsigned k = gtid; k < P.np; k += gstride) {
                if (nl) nl_build_particle(P, S, k);
                ContactOut c;
                if (!contact_particle<PREC, MODEL>(P, S, k, srow, B, t, c)) continue;
                contact_writeback(P, S, k, c);
                integrate_particle(P, S, k, make_double4(c.F.x, c.F.y, c.F.z, 0.0f),
                                   make_double4(c.T.x, c.T.y, c.T.z, 0.0f), clk, S.x_nx, S.vel_nx,
                                   S.angvel_nx, S.vel_f_nx, S.angvel_f_nx, fr, fn);
            }
            if (!bar()) return;
            // ---- W: wall-force partials ----
            // the previous step's flags: every block read them before this barrier
            if (rank == 0 && t == 0) {
                pc->flag_resort[(iter + 1) & 1] = 0;
                pc->flag_nl[(iter + 1) & 1] = 0;
            }
            if (P.nw > 0)
                for (unsigned j = rank; j < box.nblk; j += gsz) {
                    double sj = chunk_tree_sum(S.walls_force_pp, P.np, j, cache);
                    if (t == 0) S.partials[j] = sj;
                }
            if (!bar()) return;
            // ---- every block: ordered wall sum, walls, clock, next flags ----
            double wforce = P.nw > 0 ? ordered_sum(S.partials, box.nblk, stage) : 0.0;
            if (t == 0) {
                DevCtl *ctl = S.ctl;
                walls_integrate(P, S, wforce, iter, h.t_current);   // this block's copies
                const int err = *(volatile int *)&ctl->err;
                const int nres = *(volatile int *)fr, nnl = *(volatile int *)fn;
                const double t_next = h.t_current + P.dt;
                const int vs_next = next_velocity_state(h.velocity_state, h.t_current);
                if (rank == 0) {
                    for (unsigned w = 0; w < P.nw && w < 6; ++w) {
                        g_wnx[w] = sw_nx[w];
                        g_wmvfd[w] = sw_mvfd[w];
                        g_wacc[w] = sw_acc[w];
                    }
                    ctl->iter = iter + 1;
                    ctl->t_current = t_next;
                    ctl->velocity_state = vs_next;
                    // flags the host raised were consumed by the first step;
                    // the ones raised in this step are pending for the next
                    ctl->resort = nres;
                    ctl->nl_rebuild = nnl;
                    if (resorted) ctl->resorts += 1;
                    if (nl) ctl->nl_builds += 1;
                    pc->view = v ^ 1;
                    if (err) atomicOr(A.any_err, 1);
                    __threadfence();
                }
                h.iter = iter + 1;
                h.t_current = t_next;
                h.velocity_state = vs_next;
                h.err = err;
                h.resort = nres;
                h.nl = nnl;
                h.view = v ^ 1;
            }
            __syncthreads();
        }
    }
}

}  // namespace sphb
