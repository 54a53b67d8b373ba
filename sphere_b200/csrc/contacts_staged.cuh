// Contact search and forces with the neighbour cells staged in shared memory
// (topology, src/contactsearch.cuh:194-371, and interact,
// src/contactsearch.cuh:385-726, for contact model 2).
//
// A block owns B consecutive particles of the cell sort.  Its particles lie
// in one contiguous range of cells, so every neighbour of them lies in the
// nine cell rows (dz, dy) in {-1,0,1}^2 shifted from that range (plus wrapped
// images at periodic faces).  Because particles are stored sorted by cell,
// each row is one contiguous range of sorted positions: the block copies
// those ranges (positions, velocities, angular velocities, original indices)
// into shared memory with coalesced loads, and the per-particle walk of the
// neighbour list and of the history slots then reads partners from shared
// memory instead of chasing them through global memory.  Partners outside
// the staged ranges (periodic images across a face, or ranges cut by the
// shared-memory capacity) are read from global memory.
//
// The arithmetic and its order are those of contact_particle<PREC, 2>:
// topology visits the list in the reference's order with the reference's
// slot policy; interact walks the occupied slots in slot order.  A slot that
// topology did not hit in this step is released without evaluating it: its
// partner has no image within contact distance (the list holds every pair
// within r_a + r_b + skin, or the 27-cell scan visits every image), so the
// reference's interact would find a non-negative overlap and release it too.
// Hit slots remember the list entry that hit them (partner sorted position
// and periodic shift), which replaces the reference's distmod lookup and the
// original-to-sorted indirection.
#pragma once

#include "dem_device.cuh"

namespace sphb {

constexpr unsigned kStageSegMax = 9;

// The merged sorted-position ranges a block stages.
struct StageTable {
    unsigned s[kStageSegMax];    // first sorted position
    unsigned len[kStageSegMax];  // staged count (after the capacity cut)
    unsigned off[kStageSegMax];  // first shared-memory slot
    unsigned nseg, total;
};

template <int PREC>
struct StageVel {
    using T = double4;
};
template <>
struct StageVel<2> {
    using T = float4;
};

// Read-only (non-coherent) load of a double4: the arrays read this way are
// not written by the kernel that reads them.
__device__ __forceinline__ double4 ldg4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Shared-memory bytes per staged particle.
template <int PREC>
__host__ __device__ constexpr size_t stage_bytes_per_particle()
{
    return sizeof(double4) + 2 * sizeof(typename StageVel<PREC>::T) + sizeof(uint32_t);
}

// The merged ranges of the block [k0, k1) (cells cell_of[k0] ..
// cell_of[k1 - 1]) cut at `cap` particles.  Threads 0..8 each find one of
// the nine (dz, dy) row ranges in parallel; thread 0 merges them.  Called by
// every thread of the block; T is valid after it returns.
__device__ __forceinline__ void stage_table_build(const DevParams &P, const DevState &S,
                                                  unsigned k0, unsigned k1, unsigned cap,
                                                  StageTable &T)
{
    __shared__ unsigned row_lo[kStageSegMax], row_hi[kStageSegMax];
    const unsigned t = threadIdx.x;
    if (t < kStageSegMax) {
        const long long nx = P.num[0], nxy = (long long)P.num[0] * P.num[1];
        const long long ncell = P.ncells;
        const long long cf = __ldg(&S.cell_of[k0]), cl = __ldg(&S.cell_of[k1 - 1]);
        const int dz = (int)(t / 3) - 1, dy = (int)(t % 3) - 1;
        long long a = cf + dz * nxy + dy * nx - 1, b = cl + dz * nxy + dy * nx + 1;
        if (a < 0) a = 0;
        if (b > ncell - 1) b = ncell - 1;
        unsigned lo = 0, hi = 0;
        if (a <= b) {
            lo = a == 0 ? 0u : __ldg(&S.cell_end[a - 1]);
            hi = __ldg(&S.cell_end[b]);
        }
        row_lo[t] = lo;
        row_hi[t] = hi > lo ? hi : lo;
    }
    __syncthreads();
    if (t == 0) {
        unsigned s[kStageSegMax], e[kStageSegMax];
        unsigned n = 0;
        for (unsigned r = 0; r < kStageSegMax; ++r) {
            const unsigned lo = row_lo[r], hi = row_hi[r];
            if (hi <= lo) continue;
            unsigned j = n++;
            while (j > 0 && s[j - 1] > lo) {
                s[j] = s[j - 1];
                e[j] = e[j - 1];
                --j;
            }
            s[j] = lo;
            e[j] = hi;
        }
        unsigned m = 0;
        for (unsigned i = 0; i < n; ++i) {
            if (m > 0 && s[i] <= e[m - 1]) {
                if (e[i] > e[m - 1]) e[m - 1] = e[i];
            } else {
                s[m] = s[i];
                e[m] = e[i];
                ++m;
            }
        }
        unsigned total = 0, nseg = 0;
        for (unsigned i = 0; i < m && total < cap; ++i) {
            const unsigned len = min(e[i] - s[i], cap - total);
            T.s[nseg] = s[i];
            T.len[nseg] = len;
            T.off[nseg] = total;
            ++nseg;
            total += len;
        }
        T.nseg = nseg;
        T.total = total;
    }
    __syncthreads();
}

// Shared-memory slot of sorted position b, or -1 when it is not staged.
__device__ __forceinline__ int stage_lookup(const StageTable &T, unsigned b)
{
    for (unsigned r = 0; r < T.nseg; ++r) {
        const unsigned d = b - T.s[r];
        if (d < T.len[r]) return (int)(T.off[r] + d);
    }
    return -1;
}

template <int PREC>
struct StageView {
    using V = typename StageVel<PREC>::T;
    double4 *x;
    V *vel, *angvel;
    uint32_t *orig;
};

// Carves the dynamic shared memory: srow and the hit entries (nc * B each),
// then the staged arrays of `cap` particles.
template <int PREC>
__device__ __forceinline__ StageView<PREC> stage_carve(unsigned char *base, unsigned nc, unsigned B,
                                                       unsigned cap, uint32_t *&srow,
                                                       uint32_t *&shit)
{
    using V = typename StageVel<PREC>::T;
    srow = reinterpret_cast<uint32_t *>(base);
    shit = srow + (size_t)nc * B;
    unsigned char *p = reinterpret_cast<unsigned char *>(shit + (size_t)nc * B);
    StageView<PREC> v;
    v.x = reinterpret_cast<double4 *>(p);
    p += (size_t)cap * sizeof(double4);
    v.vel = reinterpret_cast<V *>(p);
    p += (size_t)cap * sizeof(V);
    v.angvel = reinterpret_cast<V *>(p);
    p += (size_t)cap * sizeof(V);
    v.orig = reinterpret_cast<uint32_t *>(p);
    return v;
}

__host__ __device__ constexpr size_t stage_smem_bytes(size_t nc, size_t B, size_t cap,
                                                      size_t per_particle)
{
    return 2 * nc * B * sizeof(uint32_t) + cap * per_particle;
}

// Copies the staged ranges into shared memory (all threads of the block),
// four particles per thread in flight.
template <int PREC>
__device__ __forceinline__ void stage_fill(const DevState &S, const StageTable &T,
                                           const StageView<PREC> &V)
{
    using VT = typename StageVel<PREC>::T;
    const unsigned total = T.total, B = blockDim.x;
    for (unsigned i0 = threadIdx.x; i0 < total; i0 += 4 * B) {
        double4 x[4];
        VT v[4], w[4];
        uint32_t o[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const unsigned i = i0 + q * B;
            if (i < total) {
                unsigned r = 0;
                while (r + 1 < T.nseg && i >= T.off[r + 1]) ++r;
                const unsigned b = T.s[r] + (i - T.off[r]);
                x[q] = ldg4(&S.x[b]);
                if constexpr (PREC == 2) {
                    v[q] = __ldg(&S.vel_f[b]);
                    w[q] = __ldg(&S.angvel_f[b]);
                } else {
                    v[q] = ldg4(&S.vel[b]);
                    w[q] = ldg4(&S.angvel[b]);
                }
                o[q] = __ldg(&S.orig_of[b]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const unsigned i = i0 + q * B;
            if (i < total) {
                V.x[i] = x[q];
                V.vel[i] = v[q];
                V.angvel[i] = w[q];
                V.orig[i] = o[q];
            }
        }
    }
}

// Contact search and forces of sorted particle k.  srow / shit are this
// thread's slot partner ids and hit entries in shared memory (slot i at
// [i * B + t]).  With STAGE the partners come from the staged ranges where
// they are staged; otherwise (or outside them) from global memory.  The
// neighbour-list entries and their partners' positions are fetched eight at
// a time, and the partners of hit slots IB at a time, so the loads of a batch
// are in flight together; the visits and the force sums keep their order.
// Returns false after raising a capacity error.
template <int PREC, bool STAGE, int IB>
__device__ __forceinline__ bool contact_particle_staged(const DevParams &P, const DevState &S,
                                                        unsigned k, const StageTable &T,
                                                        const StageView<PREC> &V, uint32_t *srow,
                                                        uint32_t *shit, unsigned B, unsigned t,
                                                        ContactOut &out)
{
    using VT = typename StageVel<PREC>::T;
    constexpr int TP = PREC == 2 ? 1 : PREC;  // precision of overlap tests
    const unsigned NC = P.nc;
    const uint64_t full = NC >= 64 ? ~0ull : ((1ull << NC) - 1ull);
    const unsigned o = __ldg(&S.orig_of[k]);
    const double4 xa = ldg4(&S.x[k]);
    const double ra = xa.w;
    const double4 vel_a = ldg4(&S.vel[k]);
    const V3 angvel_a = xyz(ldg4(&S.angvel[k]));
    double es_dot = 0.0, ev_dot = 0.0, p = 0.0;
    V3 F = mk3(0.0, 0.0, 0.0), T3 = mk3(0.0, 0.0, 0.0);
    const unsigned cnt = __ldg(&S.nl_count[k]);
    const size_t np = P.np;
    const size_t rowbase = (size_t)o * NC;
    uint64_t mask = S.occ[o];
    uint64_t written = 0, hit = 0;
    {
        uint64_t m = mask;
        while (m) {
            int i = __ffsll((long long)m) - 1;
            srow[i * B + t] = S.contacts[rowbase + i];
            m &= m - 1;
        }
    }
    // --- topology ---
    int nc = 0;
    bool ok = true;
    // visit of list entry e whose partner b sits at shared slot si (or -1)
    // with position xb
    auto visit = [&](uint32_t e, int si, const double4 &xb) {
        const unsigned b = e & 0x0fffffffu;
        const double rb = xb.w;
        const uint32_t c = e >> 28;
        const int sx = (c & 1) ? 1 : ((c & 2) ? -1 : 0);
        const int sy = (c & 4) ? 1 : ((c & 8) ? -1 : 0);
        V3 xab = mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
        xab = add3(xab, shift_vec(P, sx, sy));
        const double len = vlen<TP>(xab);
        const double delta = len - (ra + rb);
        if (delta < 0.0) {
            const unsigned b_orig = si >= 0 ? V.orig[si] : __ldg(&S.orig_of[b]);
            const int cpos = pick_slot(mask, full, srow, B, t, b_orig, nc);
            if (cpos >= (int)NC || nc + 1 > (int)NC) {
                raise_err(S.ctl, DERR_CAPACITY, (int)o);
                ok = false;
                return;
            }
            srow[cpos * B + t] = b_orig;
            shit[cpos * B + t] = e;
            mask |= 1ull << cpos;
            written |= 1ull << cpos;
            hit |= 1ull << cpos;
            S.dmcode[rowbase + cpos] = (uint8_t)c;
            ++nc;
        }
    };
    auto slot_of = [&](unsigned b) -> int {
        if constexpr (STAGE) return stage_lookup(T, b);
        else return -1;
    };
    if (cnt != NL_OVERFLOW) {
        for (unsigned j0 = 0; j0 < cnt && ok; j0 += 8) {
            uint32_t ev[8];
            int si[8];
            double4 xb[8];
#pragma unroll
            for (unsigned q = 0; q < 8; ++q)
                ev[q] = j0 + q < cnt ? __ldg(&S.nl[(size_t)(j0 + q) * np + k]) : 0u;
#pragma unroll
            for (unsigned q = 0; q < 8; ++q) {
                si[q] = -1;
                if (j0 + q < cnt) {
                    const unsigned b = ev[q] & 0x0fffffffu;
                    si[q] = slot_of(b);
                    xb[q] = si[q] >= 0 ? V.x[si[q]] : ldg4(&S.x[b]);
                }
            }
#pragma unroll
            for (unsigned q = 0; q < 8; ++q)
                if (j0 + q < cnt && ok) visit(ev[q], si[q], xb[q]);
        }
    } else {
        for_each_cell_candidate(P, S, k, xa, [&](unsigned b, int sx, int sy) -> bool {
            const int si = slot_of(b);
            const double4 xb = si >= 0 ? V.x[si] : ldg4(&S.x[b]);
            visit(b | ((uint32_t)dm_encode(sx, sy) << 28), si, xb);
            return ok;
        });
    }
    if (!ok) return false;
    // --- interact ---
    // occupied slots that topology did not hit: released (their partner has
    // no image within contact distance)
    {
        uint64_t rel = mask & ~hit;
        while (rel) {
            const int i = __ffsll((long long)rel) - 1;
            rel &= rel - 1;
            mask &= ~(1ull << i);
            written |= 1ull << i;
            if constexpr (PREC == 2) S.delta_t_f[rowbase + i] = make_float4(0.f, 0.f, 0.f, 0.f);
            else S.delta_t[rowbase + i] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
    }
    // hit slots in slot order (the reference's summation order), IB at a time
    uint64_t hm = hit;
    while (hm) {
        int sl[IB], si[IB];
        unsigned kb[IB];
        double4 xb[IB];
        VT vb[IB], wb[IB];
        uint32_t code[IB];
        float4 hf[IB];
        double4 hd[IB];
#pragma unroll
        for (int q = 0; q < IB; ++q) {
            sl[q] = -1;
            if (hm) {
                const int i = __ffsll((long long)hm) - 1;
                hm &= hm - 1;
                sl[q] = i;
                const uint32_t e = shit[i * B + t];
                kb[q] = e & 0x0fffffffu;
                code[q] = e >> 28;
                si[q] = slot_of(kb[q]);
                if (si[q] >= 0) {
                    xb[q] = V.x[si[q]];
                    vb[q] = V.vel[si[q]];
                    wb[q] = V.angvel[si[q]];
                } else {
                    xb[q] = ldg4(&S.x[kb[q]]);
                    if constexpr (PREC == 2) {
                        vb[q] = __ldg(&S.vel_f[kb[q]]);
                        wb[q] = __ldg(&S.angvel_f[kb[q]]);
                    } else {
                        vb[q] = ldg4(&S.vel[kb[q]]);
                        wb[q] = ldg4(&S.angvel[kb[q]]);
                    }
                }
                if constexpr (PREC == 2) hf[q] = S.delta_t_f[rowbase + i];
                else hd[q] = S.delta_t[rowbase + i];
            }
        }
#pragma unroll
        for (int q = 0; q < IB; ++q) {
            if (sl[q] < 0) continue;
            const size_t mempos = rowbase + sl[q];
            const V3 dm = dm_decode(P, (uint8_t)code[q]);
            const double rb = xb[q].w;
            const V3 x_ab = mk3(xa.x - xb[q].x + dm.x, xa.y - xb[q].y + dm.y,
                                xa.z - xb[q].z + dm.z);
            const double len = vlen<TP>(x_ab);
            const double delta_n = len - (ra + rb);
            if constexpr (PREC == 2) {
                float4 h = hf[q];
                mixed_pair(P, F, T3, es_dot, ev_dot, p, __ldg(&S.vel_f[k]), __ldg(&S.angvel_f[k]),
                           vb[q], wb[q], h, ra, rb, x_ab, len, delta_n);
                S.delta_t_f[mempos] = h;
            } else {
                V3 dt_new = contact_linear<PREC>(P, F, T3, es_dot, ev_dot, p, vel_a, angvel_a,
                                                 vb[q], xyz(wb[q]), hd[q], ra, rb, x_ab, len,
                                                 delta_n);
                S.delta_t[mempos] = make_double4(dt_new.x, dt_new.y, dt_new.z, 0.0);
            }
        }
    }
    if (written) {
        uint64_t w = written;
        while (w) {
            int i = __ffsll((long long)w) - 1;
            w &= w - 1;
            S.contacts[rowbase + i] = (mask >> i) & 1ull ? srow[i * B + t] : P.np;
        }
        S.occ[o] = mask;
    }
    contact_walls<PREC>(P, S, xa, ra, vel_a, angvel_a, F, T3, es_dot, ev_dot, p, out);
    return true;
}

// Threads per block of the staged contact kernel and resident blocks per SM;
// SPHB_STAGED_ON = 0 builds it without the shared-memory staging (partners
// from global memory, batched loads only).
#ifndef SPHB_STAGED_B
#define SPHB_STAGED_B 128
#endif
#ifndef SPHB_STAGED_MINB
#define SPHB_STAGED_MINB 2
#endif
#ifndef SPHB_STAGED_ON
#define SPHB_STAGED_ON 1
#endif
// partners of hit slots fetched together
#ifndef SPHB_STAGED_IB
#define SPHB_STAGED_IB 4
#endif

template <int PREC>
__global__ void __launch_bounds__(SPHB_STAGED_B, SPHB_STAGED_MINB)
    k_contacts_staged(DevParams P, DevState S, unsigned cap)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StageTable T;
    const unsigned B = blockDim.x, t = threadIdx.x;
    const unsigned k0 = blockIdx.x * B;
    const unsigned k1 = min(k0 + B, P.np);
    const unsigned k = k0 + t;
    if (k == 0 && S.ctl->nl_rebuild) S.ctl->nl_rebuild = 0;  // k_resort has rebuilt the lists
    uint32_t *srow, *shit;
    const StageView<PREC> V = stage_carve<PREC>(smem_raw, P.nc, B, cap, srow, shit);
    if (SPHB_STAGED_ON && cap > 0) {
        stage_table_build(P, S, k0, k1, cap, T);
        stage_fill<PREC>(S, T, V);
    }
    if (S.ctl->err || k >= P.np) return;
    ContactOut c;
    constexpr int IB = PREC == 2 ? SPHB_STAGED_IB : (SPHB_STAGED_IB > 2 ? 2 : SPHB_STAGED_IB);
    if (!contact_particle_staged<PREC, (bool)SPHB_STAGED_ON, IB>(P, S, k, T, V, srow, shit, B, t,
                                                                  c))
        return;
    contact_writeback(P, S, k, c);
}

}  // namespace sphb
