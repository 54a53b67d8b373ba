/*
 * sphere_b200 -- C ABI of the B200 DEM step engine.
 *
 * The engine replaces what `sim.run()` reaches through a subprocess in the
 * reference (python/sphere.py:4482-4540 -> src/main.cpp:28-211 ->
 * DEM::DEM + DEM::startTime, src/sphere.cpp:16-95, src/device.cu:833-2834).
 * Plain pointers and sizes only; every call returns a status code (0 = OK,
 * < 0 = error, > 0 = warning) instead of exiting the process as the
 * reference does (src/utility.cu:11-60).
 *
 * Ownership: the engine owns all device memory and its CUDA stream; callers
 * own paths and host buffers.  A handle is used by one host thread at a time.
 */
#ifndef SPHERE_B200_H_
#define SPHERE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sph_engine sph_engine;

/* Status codes. */
enum {
    SPH_OK = 0,
    SPH_WARN_NOCONV = 1,        /* Darcy solve hit maxiter (the reference continues) */
    SPH_ERR_FILE = -1,          /* cannot open / short read / trailing bytes */
    SPH_ERR_VERSION = -2,       /* format version is not 2.15 (src/file_io.cpp:47-54) */
    SPH_ERR_INPUT = -3,         /* value check failed (src/sphere.cpp:145-345) */
    SPH_ERR_CUDA = -4,          /* CUDA runtime error */
    SPH_ERR_OUTSIDE = -5,       /* particle left the grid or became non-finite */
    SPH_ERR_CAPACITY = -6,      /* contact slots exhausted (the reference drops silently) */
    SPH_ERR_UNSUPPORTED = -7,   /* input uses a path this engine does not build */
    SPH_ERR_ARG = -8,           /* bad argument / buffer size */
    SPH_ERR_TIMEOUT = -9,       /* a bounded device wait gave up */
};

/* Arithmetic of the DEM step. */
enum {
    SPH_PREC_FAITHFUL = 0, /* FP64 with the reference's FP32 vector lengths */
    SPH_PREC_FP64 = 1,     /* FP64 throughout (FP64 square roots) */
    SPH_PREC_MIXED = 2,    /* FP32 contact kinematics and forces, FP64 overlap,
                              accumulators, integration and reductions */
};

typedef struct sph_opts {
    size_t struct_size;   /* sizeof(sph_opts) as the caller compiled it.  Set it before
                             calling sph_default_opts; sph_default_opts and every call
                             that takes options refuse any other value with
                             SPH_ERR_ARG, so a caller built against another layout of
                             this struct cannot make the library read or write past
                             the caller's copy */
    int fluid;            /* 1: the file has a fluid section (the reference's --fluid) */
    int device;           /* CUDA device ordinal; -1 keeps the current device */
    int verbose;          /* 1: progress on stdout like DEM::startTime */
    int precision;        /* SPH_PREC_* */
    int integrator;       /* 3: three-term Taylor (the reference's TY3), 2: two-term */
    int contact_capacity; /* contact slots per particle; the reference's NC is 32 */
    int warm_start;       /* Darcy start: 0 the previous solution (the reference's),
                             1 learned (a network's correction of the cubic
                             extrapolation in time of the last four solutions,
                             or that extrapolation alone, whichever has the
                             smaller first residual), 2 that extrapolation
                             alone; 1 and 2 fall back to the previous solution
                             when its first residual is smaller */
    int graph_steps;      /* DEM steps captured per CUDA graph launch; 0 = automatic */
    const char *output_dir; /* directory for .bin/status/conv outputs; NULL = "output" */
    int step_kernel;      /* 0 automatic (the fused persistent step where it applies),
                             1 per-stage kernels, 2 fused persistent step (error where
                             it does not apply: bonds, fluid, wmode 3), 3 per-stage
                             kernels with the contact search reading its partners
                             from the neighbour cells staged in shared memory
                             (same results; slower on the measured workloads),
                             4 per-stage kernels with the contact search and the
                             particle integration in one launch, integrating into
                             a second buffer of x / vel / angvel (same results;
                             error where it does not apply: bonds, fluid, wmode 3) */
    int darcy_exact_stop; /* 1: the Darcy Jacobi loop tests the residual at every
                             iteration and stops at the first that meets the
                             tolerance; 0 (default): the reference's test at
                             iterations 0, 10, 20, ... (src/device.cu:2340-2366) */
    int inject_timeout;   /* test knob, 0 in normal use: a mask of SPH_INJECT_*.  The
                             bounded device waits of the selected cooperative kernels
                             then wait for a value that nothing writes and give up
                             after about a thousand polls, so the step returns
                             SPH_ERR_TIMEOUT; this exercises the timeout path without
                             a GPU fault.  An engine that timed out is closed. */
} sph_opts;

/* Kernels whose waits sph_opts.inject_timeout makes time out. */
enum {
    SPH_INJECT_RESORT = 1,     /* the grid barrier of the cooperative cell re-sort */
    SPH_INJECT_PERSISTENT = 2, /* the group barrier of the fused persistent step */
    SPH_INJECT_DARCY = 4,      /* the neighbour waits of the Darcy Jacobi kernel */
    SPH_INJECT_NS = 8,         /* the barrier and waits of the Navier-Stokes Jacobi kernel */
};

/* Fields for sph_get/sph_set.  Vector fields use the reference's Float4
 * layout (4 doubles per particle, src/datatypes.h:16-33) in ORIGINAL
 * particle order, so results compare directly with the reference's arrays. */
typedef enum sph_field {
    SPH_F_X = 0,        /* np x (x, y, z, radius) */
    SPH_F_VEL,          /* np x (vx, vy, vz, fixvel) */
    SPH_F_ANGVEL,       /* np x (wx, wy, wz, 0) */
    SPH_F_ANGPOS,
    SPH_F_FORCE,
    SPH_F_TORQUE,
    SPH_F_ACC,
    SPH_F_ANGACC,
    SPH_F_XYZSUM,
    SPH_F_ES_DOT,       /* np doubles */
    SPH_F_ES,
    SPH_F_EV_DOT,
    SPH_F_EV,
    SPH_F_P,
    SPH_F_CELLID,       /* np u32: sorted cell keys (thrust::sort_by_key output) */
    SPH_F_INDEX,        /* np u32: original index of each sorted position */
    SPH_F_CELLSTART,    /* ncells u32, 0xffffffff for empty cells */
    SPH_F_CELLEND,      /* ncells u32 (valid where cellstart is not empty) */
    SPH_F_CONTACTS,     /* np*capacity u32, keyed by original index; np = empty */
    SPH_F_DELTA_T,      /* np*capacity x 4 doubles: tangential history */
    SPH_F_DISTMOD,      /* np*capacity x 4 doubles: periodic shift + partner radius */
    SPH_F_WALLS_NX,     /* nw x (nx, ny, nz, position) */
    SPH_F_WALLS_MVFD,   /* nw x (mass, velocity, force, sigma0) */
    SPH_F_WALLS_ACC,    /* nw doubles */
    SPH_F_ITER,         /* 1 int64: DEM steps taken */
    SPH_F_TIME,         /* 1 double: model time */
    SPH_F_DARCY_P,      /* nx*ny*nz doubles, x fastest */
    SPH_F_DARCY_PHI,
    SPH_F_DARCY_DPHI,
    SPH_F_DARCY_K,
    SPH_F_DARCY_V,      /* nx*ny*nz x 3 doubles */
    SPH_F_DARCY_F_P,    /* np x 4 doubles: pressure force on each particle */
    SPH_F_DARCY_ITERS,  /* 1 int64: Jacobi iterations of the last fluid step */
    SPH_F_DARCY_ITERS_TOTAL, /* 1 int64: Jacobi iterations since open */
    SPH_F_DARCY_ITERS_EXACT, /* 1 int64: first iteration of the last solve whose
                                residual met the tolerance (-1: none) */
    SPH_F_DARCY_WARM,   /* 4 x 8 bytes: warm-start predictions, training steps,
                           solves started from the network's guess (int64),
                           last training loss (double) */
    SPH_F_BONDS,        /* nb0 x 2 u32 */
    SPH_F_BONDS_DELTA,  /* nb0 x 4 doubles (t.x, t.y, t.z, n) */
    SPH_F_BONDS_OMEGA,
    SPH_F_VELOCITY_STATE, /* 1 int64: rate-state velocity step state (device.cu:2461-2469) */
    /* Navier-Stokes runs (cfd_solver 0) also answer the SPH_F_DARCY_P, _PHI,
     * _DPHI, _V (cell-centre velocity), _F_P (pressure force), _ITERS and
     * _ITERS_TOTAL fields above (navierstokes.cuh device arrays) */
    SPH_F_NS_EPSILON,   /* nx*ny*nz doubles: pressure change of the last projection */
    SPH_F_NS_NORM,      /* nx*ny*nz doubles: normalised Jacobi residuals */
    SPH_F_NS_V_FACE,    /* (nx+1)(ny+1)(nz+1) x 3 doubles: staggered face velocities
                           v_x, v_y, v_z at faces 0..n per axis, x fastest */
    SPH_F_NS_F_D,       /* np x 4 doubles: drag force on each particle */
    SPH_F_NS_F_V,       /* np x 4 doubles: viscous force */
    SPH_F_NS_F_SUM,     /* np x 4 doubles: total fluid force */
    SPH_F_COUNT
} sph_field;

typedef struct sph_info {
    uint32_t np, nw, nb0, capacity;
    uint32_t num[3];
    int32_t periodic, contactmodel, precision, fluid;
    int64_t iter;
    double time, time_total, dt, file_dt;
    uint32_t step_count;
    int64_t resorts;      /* re-sorts performed (steps where a particle changed cell) */
    int32_t step_path;    /* 0 per-stage kernels, 1 fused persistent step, 2 per-stage
                             kernels with contacts and integration in one launch */
    int32_t step_threads; /* persistent path: threads per block chosen by the autotuner */
    int32_t step_grid;    /* persistent path: blocks of the launch */
    int32_t tuned;        /* 1 once the autotuner has run */
} sph_info;

/* Fills *opts with the defaults (faithful FP64, TY3, 32 slots, device -1).
 * The caller sets opts->struct_size = sizeof(sph_opts) first; any other
 * value returns SPH_ERR_ARG and writes nothing. */
int sph_default_opts(sph_opts *opts);

/* Reads and validates a .bin file without touching the device: the
 * reference's `sphere --dry` (src/sphere.cpp:46-51: read, checkValues,
 * report, exit).  The message of a failure is in sph_open_error(). */
int sph_check_file(const char *bin_path, int fluid);

/* Reads and validates a .bin file (src/file_io.cpp:30-417 +
 * src/sphere.cpp:145-345) and uploads the state.  Replaces `DEM dem(...)`
 * at src/main.cpp:184. */
int sph_open(const char *bin_path, const sph_opts *opts, sph_engine **out);

/* Same as sph_open, from the bytes of a .bin file held in host memory. */
int sph_open_buffer(const void *bytes, size_t nbytes, const sph_opts *opts,
                    const char *sid, sph_engine **out);

/* The full time loop with the reference's side effects: output files
 * <out>/<sid>.output%05d.bin every file_dt, <sid>.status.dat, and
 * <sid>-conv.log when fluid.  Replaces DEM::startTime (src/device.cu:833). */
int sph_run(sph_engine *e);

/* Advances n DEM steps without file output (benchmarks, parity tests). */
int sph_step(sph_engine *e, uint64_t n);

/* Same as sph_step; *device_ms receives the device time of the n steps,
 * measured with CUDA events recorded on the engine's stream. */
int sph_step_timed(sph_engine *e, uint64_t n, double *device_ms);

/* Per-kernel device time of the step, averaged over n DEM steps run
 * eagerly with CUDA events around each stage (the reference's PROFILING
 * table, src/device.cu:954-994,2717-2815).  The steps advance the run. */
typedef struct sph_profile {
    double resort_ms;     /* cell re-sort (skipped when no cell changed) */
    double contacts_ms;   /* contact search + contact/wall forces */
    double bonds_ms;      /* bond forces */
    double fluid_ms;      /* Darcy solver */
    double integrate_ms;  /* integration + wall reduction + wall update */
    double step_ms;       /* whole step */
    uint64_t steps;
} sph_profile;
int sph_profile_steps(sph_engine *e, uint64_t n, sph_profile *out);

/* Number of bytes sph_get/sph_set move for a field (0 if not present). */
int64_t sph_field_bytes(sph_engine *e, sph_field f);

/* Copies a field to host memory (synchronises the engine's stream). */
int sph_get(sph_engine *e, sph_field f, void *dst, size_t bytes);

/* Overwrites a field from host memory (positions, velocities, ...);
 * returns once the source buffer has been read.  New positions take effect
 * at the next step, which re-sorts and rebuilds the neighbour lists where a
 * particle changed cell, left its list skin or changed radius; a position
 * outside the grid is reported here (SPH_ERR_OUTSIDE). */
int sph_set(sph_engine *e, sph_field f, const void *src, size_t bytes);

/* Writes the current state as a .bin file (src/file_io.cpp:420-731). */
int sph_write_bin(sph_engine *e, const char *path);

int sph_get_info(sph_engine *e, sph_info *info);

/* Device time of the cell hash + stable cell sort + reorder of the current
 * state (the reference's calcParticleCellID + sort_by_key + reorderArrays,
 * src/device.cu:1066-1114), averaged over reps forced sorts.  A sort of
 * sorted particles is the identity, so the run is unchanged. */
int sph_time_sort(sph_engine *e, int reps, double *ms_per_sort);

/* Energy sum of the current state, computed on the device.  Replaces
 * sim.energy(method) (python/sphere.py:4311-4380); method is one of "pot",
 * "kin", "rot", "shear", "shearrate", "visc_n", "visc_n_rate", "bondpot"
 * with the reference's formulas (its "bondpot" multiplies each bond's
 * tangential factors by the norm of the whole delta_t / omega_t arrays,
 * and so does this).  An unknown method is SPH_ERR_ARG, as the reference
 * raises. */
int sph_energy(sph_engine *e, const char *method, double *out);

/* Porosity in z_slices horizontal slabs from z = 0 to the upper wall
 * (L_z without walls); z_pos and porosity receive z_slices values each.
 * Replaces DEM::porosity (src/sphere.cpp:487-605), the `porosity` program
 * behind sim.porosity() (python/sphere.py:4437-4480), with its case
 * analysis and its slice-height check against twice the radius of the
 * last particle (SPH_ERR_ARG where the reference exits). */
int sph_porosity(sph_engine *e, int z_slices, double *z_pos, double *porosity);

/* Overlapping particle pairs: i < j (original indices), separation
 * |x_j - x_i| - (r_i + r_j) < 0, both fixvel flags zero, no periodic
 * images -- the list of DEM::findOverlaps (src/sphere.cpp:677-725) that
 * `sphere --contacts` prints (src/sphere.cpp:904-913) for
 * sim.findOverlaps() (python/sphere.py:4868-4883), in the same order
 * (i, then j ascending) with the same FP64 separations.  *count receives
 * the number of pairs.  With pairs and delta NULL only the count is
 * computed; otherwise pairs (2 x capacity u32) and delta (capacity
 * doubles) are filled, or SPH_ERR_ARG is returned when capacity < count. */
int sph_overlaps(sph_engine *e, uint32_t *pairs, double *delta, uint64_t capacity,
                 uint64_t *count);

/* Ray-traced image of the current state into rgba (width x height x 4
 * bytes, pixel i + j * width, alpha 255), replacing DEM::render
 * (src/raytracer.cuh: rayInitPerspective, rayIntersectSpheres and
 * rayIntersectSpheresColormap with the camera of DEM::cameraInit) behind
 * `sphere --render`; the caller writes the PPM (DEM::writePPM,
 * src/file_io.cpp:734-757).  method 0: shaded spheres; 1 pressure,
 * 2 speed, 3 angular speed, 4 x displacement, 5 rotation, coloured over
 * [0, max_val] (fixed particles grey); with lower_cutoff > 0 only free
 * particles whose value exceeds it are drawn.  The reference's defaults
 * are method 1, max_val 1e3, 800 x 800. */
int sph_render(sph_engine *e, int method, float max_val, float lower_cutoff, uint32_t width,
               uint32_t height, unsigned char *rgba);

/* Message for the last non-zero status of this handle (never NULL). */
const char *sph_last_error(sph_engine *e);

/* Message for a failed sph_open (thread-local; never NULL). */
const char *sph_open_error(void);

void sph_close(sph_engine *e);

/* Cell sort without allocation.  This entry point has no counterpart in the
 * reference; it exists for callers that cannot allocate device memory --
 * for example a host application whose own memory pool owns the GPU and
 * forbids outside cudaMalloc, or a time-critical loop that must not call
 * cudaMalloc/cudaFree because those calls synchronise the device.  It
 * computes what the engine's sort computes: for np positions x4 (device
 * pointer, np x (x, y, z, radius) doubles, original order) on the grid
 * (origo, L, num), the stable cell sort -- cellid[np] sorted cell keys,
 * index[np] original indices, cell_start/cell_end[num0*num1*num2]
 * (0xffffffff start for empty cells) -- all device pointers the caller owns.
 * Its scratch is one static device array built into the library
 * (SPH_NOALLOC_MAX_CELLS cells, about 8.4 MB on every GPU that loads the
 * library, held until exit); larger grids are rejected with SPH_ERR_ARG.
 * The first call on a device looks the array up on that device
 * (cudaGetSymbolAddress); later calls reuse it.  Every call shares that one
 * array, so calls whose work overlaps on the GPU (another stream, another
 * thread) race: serialise them.  `stream` is a cudaStream_t (NULL = legacy
 * default stream); the call waits for its own work.  A cell holding more
 * than SPH_NOALLOC_MAX_PER_CELL particles (a grid far coarser than a contact
 * search uses) is rejected with SPH_ERR_ARG rather than ordered by a slow
 * loop.  Returns SPH_OK, SPH_ERR_ARG, SPH_ERR_OUTSIDE (a position outside
 * the grid) or SPH_ERR_CUDA; sph_noalloc_error() describes the calling
 * thread's last failure (the message is thread-local). */
#define SPH_NOALLOC_MAX_CELLS (1u << 20)
#define SPH_NOALLOC_MAX_PER_CELL 512u
int sph_sort_cells_noalloc(const double *x4, uint32_t np, const double origo[3],
                           const double L[3], const uint32_t num[3], uint32_t *cellid,
                           uint32_t *index, uint32_t *cell_start, uint32_t *cell_end,
                           void *stream);
const char *sph_noalloc_error(void);

/* Library build string: version, arch, compile flags of the DEM kernels. */
const char *sph_version(void);

/* ---------------------------------------------------------------------
 * Batches: many independent boxes stepped by one launch of the fused
 * persistent step kernel.  Every box is a dry simulation (no fluid, no
 * bonds, no wmode-3 wall) with the same contact model and precision; boxes
 * may differ in size, parameters, walls and time step.  This replaces
 * running the reference binary once per box.
 * --------------------------------------------------------------------- */
typedef struct sph_batch sph_batch;

typedef struct sph_batch_config {
    int threads;     /* threads per block */
    int group_size;  /* blocks that step one box together */
    int grid;        /* blocks of the launch */
    int tuned;       /* 1 after the autotuner ran */
    int ntrials;     /* autotuner trials recorded */
    int graph;       /* 1 when steps replay a captured CUDA graph */
} sph_batch_config;

typedef struct sph_batch_trial {
    int threads, group_size, grid;
    double ms_per_step;   /* device time of the trial launch per step */
} sph_batch_trial;

/* Opens nbox boxes from .bin files; opts applies to every box (fluid and
 * step_kernel are ignored).  The message of a failure is in
 * sph_batch_open_error(). */
int sph_open_batch(const char *const *bin_paths, int nbox, const sph_opts *opts, sph_batch **out);
int sph_open_batch_buffers(const void *const *bufs, const size_t *sizes, int nbox,
                           const sph_opts *opts, sph_batch **out);
const char *sph_batch_open_error(void);
/* Advances every box by n steps.  The first call with at least 256 steps
 * runs the autotuner on its first steps. */
int sph_batch_step(sph_batch *b, uint64_t n);
/* Same, without tuning; *device_ms = device time (CUDA events). */
int sph_batch_step_timed(sph_batch *b, uint64_t n, double *device_ms);
/* Times every (threads, group size) on trial_steps real steps each and
 * keeps the fastest. */
int sph_batch_autotune(sph_batch *b, uint64_t trial_steps);
int sph_batch_size(sph_batch *b);
int64_t sph_batch_field_bytes(sph_batch *b, int box, sph_field f);
int sph_batch_get(sph_batch *b, int box, sph_field f, void *dst, size_t bytes);
int sph_batch_write_bin(sph_batch *b, int box, const char *path);
int sph_batch_get_config(sph_batch *b, sph_batch_config *cfg);
/* Copies up to max autotuner trials; returns how many were recorded. */
int sph_batch_get_trials(sph_batch *b, sph_batch_trial *out, int max);
const char *sph_batch_last_error(sph_batch *b);
void sph_batch_close(sph_batch *b);

/* ---------------------------------------------------------------------
 * The warm-start network alone (4 -> 16 -> 16 -> 1 channels, 3x3x3
 * kernels, ReLU; BF16 tensor-core kernels with FP32 accumulation) on host
 * arrays, for gradient checks.  The engine uses it through
 * sph_opts.warm_start.  Layer parameters: w [27 taps][16 out][16 in]
 * (taps z-major, then y, then x, offsets -1..1), b [16].  Inputs: 4
 * normalised channels per cell (x fastest: previous pressure, porosity,
 * porosity change, previous pressure change); output: channel 0 of layer 3.
 * --------------------------------------------------------------------- */
typedef struct sph_wsnet sph_wsnet;
int sph_wsnet_create(int nx, int ny, int nz, uint64_t seed, sph_wsnet **out);
int sph_wsnet_set_params(sph_wsnet *n, int layer, const float *w, const float *b);
int sph_wsnet_get_params(sph_wsnet *n, int layer, float *w, float *b);
int sph_wsnet_forward(sph_wsnet *n, const float *x4, float *out);
/* Gradients of the mean squared error over free cells (free_cells[c] != 0)
 * between the output and target: dw = 3 x [27][16][16], db = 3 x [16]. */
int sph_wsnet_gradients(sph_wsnet *n, const float *x4, const float *target,
                        const unsigned char *free_cells, float *dw, float *db);
void sph_wsnet_destroy(sph_wsnet *n);

#ifdef __cplusplus
}
#endif
#endif
