/*
 * CPU oracle for the sphere DEM step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-step algorithm (sorting,
 * contact search with history, contact/wall laws, Taylor integration, wall
 * reductions) used by the tests, smoke() and the CPU baseline of bench.py as
 * the checker.  Nothing in the product links or calls this code.
 *
 * Semantics are those of the reference kernels compiled for the host with
 * IEEE arithmetic and no contraction (-ffp-contract=off mirrors the
 * reference's --fmad=false): vector lengths are FP32 square roots of the
 * FP64 dot product in "faithful" mode (src/vector_arithmetic.h:317-324) and
 * FP64 square roots in "true FP64" mode.  Where the reference reads
 * uninitialised memory (first-step tangential history, wall mode with no
 * walls, an unassigned tangential displacement) the oracle uses zero.
 */
#ifndef SPH_ORACLE_H_
#define SPH_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

enum {
    ORC_OK = 0,
    ORC_ERR_FILE = -1,
    ORC_ERR_VERSION = -2,
    ORC_ERR_INPUT = -3,
    ORC_ERR_OUTSIDE = -4,   /* particle outside the grid / non-finite */
    ORC_ERR_CAPACITY = -5,  /* contact slot overflow */
    ORC_ERR_UNSUPPORTED = -6,
    ORC_ERR_NOCONV = -7,    /* Darcy did not converge within maxiter */
};

/* precision: 0 = faithful (FP32 lengths, as the reference), 1 = true FP64.
 * integrator: 3 = three-term Taylor (reference default), 2 = two-term.
 * nc: contact slots per particle (the reference uses 32).
 * fluid: 1 when the file holds a fluid section (the reference's --fluid). */
orc_state *orc_load(const char *path, int fluid, int precision,
                    int integrator, int nc, int *status);
void orc_free(orc_state *s);
int orc_step(orc_state *s, int64_t nsteps);
const char *orc_error(const orc_state *s);
int orc_write_bin(orc_state *s, const char *path);

/* Copies a named field into dst.  Returns bytes needed (>0) when dst is NULL
 * or too small, 0 on success, <0 for an unknown name. Names: "x", "vel",
 * "angvel", "angpos", "force", "torque", "acc", "angacc", "xyzsum" (np*4
 * doubles, the reference's Float4 layout); "es_dot", "es", "ev_dot", "ev",
 * "p" (np doubles); "cellid", "index" (np u32, sorted order); "cellstart",
 * "cellend" (ncells u32); "contacts" (np*nc u32, keyed by original index);
 * "delta_t", "distmod" (np*nc*4 doubles); "walls_nx", "walls_mvfd" (nw*4
 * doubles); "walls_acc" (nw doubles); "walls_force_partial" (nblocks
 * doubles); "darcy_p", "darcy_phi", "darcy_dphi", "darcy_k", "darcy_norm",
 * "darcy_v", "darcy_f_p"; "iter" (int64), "time" (double),
 * "darcy_nijac_last" (int64). */
int64_t orc_get(orc_state *s, const char *name, void *dst, size_t bytes);
/* Overwrites a field (same names and layouts as orc_get). */
int orc_set(orc_state *s, const char *name, const void *src, size_t bytes);

/* One stage at a time, for stage-level parity tests. */
int orc_stage_hash_sort_reorder(orc_state *s);
int orc_stage_topology(orc_state *s);
int orc_stage_interact(orc_state *s);

int orc_np(const orc_state *s);
int orc_nc(const orc_state *s);
int orc_nw(const orc_state *s);

#ifdef __cplusplus
}
#endif
#endif
