/*
 * sphgrav_b200.h -- direct-summation SPH self-gravity for NVIDIA B200 (sm_100a).
 *
 * Drop-in replacement for StarSmasher's SPHgrav_lib2 (libSPHgrav.a).  All
 * citations are paths inside the reference project.
 *
 * Physics (both precisions): every listed row i receives
 *     a_i   = sum_j  m_j f(r_ij; H_i, H_j) (x_j - x_i)
 *     phi_i = sum_j  m_j g(r_ij; H_i, H_j)
 * with H = sqrt(|range2|) = 2 hp, Newtonian when r^2 >= max(H_i^2, H_j^2) and
 * the symmetrised softening of kernel `nkernel` otherwise (0 cubic spline,
 * 1 Wendland C6, 2 Wendland C4), exactly as the reference's CPU path
 * parallel_bleeding_edge/src/cpu_grav.f:1-381 evaluates it (G = 1).
 * Point masses carry range2 < 0 (grav.f:15-18): no self-potential.
 *
 * Precisions:
 *   SPHGRAV_FP64       plain FP64 kernel; matches the CPU path to ~1e-12.
 *   SPHGRAV_F32SPLIT   positions as FP32 hi+lo pairs; pair terms in FP32 with
 *                      rsqrt.approx (variants named *_newton add one Newton
 *                      step) summed into compensated (Kahan/TwoSum) partial
 *                      sums; FP64 for the split, the cross-block partial sums,
 *                      the pairs with r < band * max H (band 1 by default,
 *                      sphgrav_set_fp64_band), the rows whose FP32 sums are
 *                      ill-conditioned (sphgrav_set_refine) and the
 *                      potential-energy diagnostic.  Max relative error of the
 *                      acceleration below 1e-6 on the benchmark workloads.
 *   SPHGRAV_TREE       Barnes-Hut octree, the approximate alternative the
 *                      reference ships with the same ABI
 *                      (misc/SPHgravtree_lib): monopole + quadrupole cells,
 *                      opening angle theta (sphgrav_set_theta, or
 *                      gpu_init_dev_'s theta for the legacy entry points;
 *                      default 0.3), softened pairs particle by particle.
 *                      Batches build one root per set (sets never interact).
 *                      Eager calls read the tree's level table and group
 *                      counts back to the host; inside a graph capture every
 *                      count stays on the device (capture after an eager call
 *                      of the same sizes, whose tree sizes the node array with
 *                      2x headroom; a replay whose tree outgrows it reports
 *                      SPHGRAV_ERR_TOO_LARGE at the next sphgrav_sync).
 *
 * Threading: a context is used by one host thread at a time.  Calls enqueue
 * work on the context's stream; functions that return results to host
 * memory synchronise that stream.
 */
#ifndef SPHGRAV_B200_H
#define SPHGRAV_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    SPHGRAV_OK = 0,
    SPHGRAV_ERR_INVALID_ARGUMENT = 1,  /* bad size, pointer, nkernel, precision */
    SPHGRAV_ERR_INVALID_INPUT = 2,     /* mass <= 0, range2 == 0, non-finite value */
    SPHGRAV_ERR_CUDA = 3,              /* CUDA runtime error (see sphgrav_last_error_message) */
    SPHGRAV_ERR_NO_DEVICE = 4,
    SPHGRAV_ERR_OUT_OF_MEMORY = 5,
    SPHGRAV_ERR_PROTOCOL = 6,          /* lasthalf without firsthalf, and similar */
    SPHGRAV_ERR_DEVICE_TIMEOUT = 7,    /* a bounded device-side wait gave up */
    SPHGRAV_ERR_TOO_LARGE = 8,         /* size beyond a documented limit */
    SPHGRAV_ERR_UNSUPPORTED = 9        /* feature not built into this library */
};

enum { SPHGRAV_FP64 = 0, SPHGRAV_F32SPLIT = 1, SPHGRAV_TREE = 2 };

typedef struct sphgrav_ctx sphgrav_ctx;
typedef struct sphgrav_graph sphgrav_graph;

/* ------------------------------------------------- legacy Fortran ABI ---
 * Same symbols, argument lists and call protocol as the reference library;
 * Fortran passes every argument by reference.  On error these log to stderr
 * and abort, as the reference's assert/exit does (cutil.h:19-27).
 * Precision: SPHGRAV_F32SPLIT unless the environment variable
 * SPHGRAV_PRECISION=fp64 (or =tree) is set or sphgrav_legacy_set_precision is
 * called.  gpu_init_dev_'s theta sets the tree mode's opening angle.
 */

/* Replaces firsthalf_grav_forces_ (grav_force_direct.cu:650-656), called from
 * grav.f:25-26, eatem.f:161 and main.f:362-374.  n particles, rows
 * [n_lower, n_lower + my_length) (1-based n_lower) are computed; q is ignored
 * like the reference's (:653-655).  Copies the inputs, enqueues the
 * computation and returns without waiting for it. */
void firsthalf_grav_forces_(int *n, int *n_lower, int *my_length,
                            double *px, double *py, double *pz,
                            double *mass, double *range2, int *q, int *nkernel);

/* Replaces lasthalf_grav_forces_ (grav_force_direct.cu:658-664), called from
 * balAV3.f:418 and eatem.f:163.  Waits for the result of the last
 * firsthalf_grav_forces_ and writes ax, ay, az, pot at the rows that call
 * listed (arrays of length n).  myrank is never read: the Fortran callers pass
 * only five arguments. */
void lasthalf_grav_forces_(int *n, double *ax, double *ay, double *az,
                           double *pot, int *myrank);

/* Replaces gpu_init_dev_ (grav_force_direct.cu:672-675), called from
 * main.f:265-275.  Selects CUDA device *myrank; theta is ignored (it is the
 * opening angle of the tree plugin). */
void gpu_init_dev_(int *myrank, double *theta);

/* Precision used by the three legacy entry points (SPHGRAV_FP64 or
 * SPHGRAV_F32SPLIT).  No reference counterpart (the reference is FP32 only,
 * grav_force_direct.cu:55-396). */
int sphgrav_legacy_set_precision(int precision);

/* ------------------------------------------------------- context API ---
 * Status-returning twins of the legacy entry points, plus the batch API.
 * No reference counterparts unless stated. */
int sphgrav_create(sphgrav_ctx **ctx, int device);
int sphgrav_destroy(sphgrav_ctx *ctx);
/* Use an existing cudaStream_t (passed as void*) instead of the context's
 * own stream; NULL restores the context's stream (pass cudaStreamLegacy,
 * (void *)1, for the legacy default stream). */
int sphgrav_set_stream(sphgrav_ctx *ctx, void *stream);
/* Wait for all work queued on the context and report a device-side error
 * (invalid input found on the device, timeout) recorded since the last call. */
int sphgrav_sync(sphgrav_ctx *ctx);

/* Status-returning twin of firsthalf_grav_forces_: host arrays of length n,
 * rows [i_begin, i_begin + ni) with 0-based i_begin. */
int sphgrav_firsthalf(sphgrav_ctx *ctx, int n, int i_begin, int ni,
                      const double *x, const double *y, const double *z,
                      const double *mass, const double *range2,
                      int nkernel, int precision);
/* Status-returning twin of lasthalf_grav_forces_: writes rows
 * [i_begin, i_begin + ni) of the host arrays (length n). */
int sphgrav_lasthalf(sphgrav_ctx *ctx, double *ax, double *ay, double *az,
                     double *pot);

/* Host-side restatement of the Fortran caller: gravforce (grav.f:12-26)
 * builds range2 = 4 hp^2, negated where u == 0, and calls firsthalf for rows
 * [ngrav_lower, ngrav_upper] (1-based, inclusive, as main.f:283-295 sets
 * them); lasthalf (balAV3.f:418) then fills gx, gy, gz, grpot at those rows.
 * Host arrays of length ntot.  Blocking. */
/* Device-resident form of sphgrav_gravforce: x, y, z, am, hp, u and the
 * outputs are device arrays of length ntot.  range2 (grav.f:15-18) is built
 * on the device into a context buffer, and rows [ngrav_lower, ngrav_upper]
 * (1-based, inclusive) of gx, gy, gz, grpot are written; the other rows are
 * left as they are.  Asynchronous on the context's stream, like
 * sphgrav_forces_device, and capturable once called with the same sizes. */
int sphgrav_gravforce_device(sphgrav_ctx *ctx, int ntot, int ngrav_lower, int ngrav_upper,
                             const double *x, const double *y, const double *z,
                             const double *am, const double *hp, const double *u,
                             int nkernel, int precision, double *gx, double *gy,
                             double *gz, double *grpot);
int sphgrav_gravforce(sphgrav_ctx *ctx, int ntot, int ngrav_lower, int ngrav_upper,
                      const double *x, const double *y, const double *z,
                      const double *am, const double *hp, const double *u,
                      int nkernel, int precision,
                      double *gx, double *gy, double *gz, double *grpot);

/* One particle set, all pointers DEVICE pointers of length n; rows
 * [i_begin, i_begin + ni) of the outputs are written.  Asynchronous on the
 * context's stream; W (device pointer to one double, may be NULL) receives
 * 0.5 * sum_rows m_i phi_i (output.f:232-252 computes it on the host). */
int sphgrav_forces_device(sphgrav_ctx *ctx, int n, int i_begin, int ni,
                          const double *x, const double *y, const double *z,
                          const double *mass, const double *range2,
                          int nkernel, int precision,
                          double *ax, double *ay, double *az, double *pot,
                          double *W);

/* Batch of independent particle sets in one persistent launch.  Set s holds
 * particles [offsets[s], offsets[s+1]) of the concatenated arrays; offsets is
 * a HOST array of nsets+1 ints.  Data pointers are DEVICE pointers.  All rows
 * of every set are computed; W_per_set (device, nsets doubles, may be NULL)
 * receives each set's 0.5 * sum m_i phi_i.  Asynchronous. */
int sphgrav_batch_forces_device(sphgrav_ctx *ctx, int nsets, const int *offsets,
                                const double *x, const double *y, const double *z,
                                const double *mass, const double *range2,
                                int nkernel, int precision,
                                double *ax, double *ay, double *az, double *pot,
                                double *W_per_set);

/* Same with HOST data pointers; copies in, computes, copies out, returns
 * when the results are in host memory. */
int sphgrav_batch_forces(sphgrav_ctx *ctx, int nsets, const int *offsets,
                         const double *x, const double *y, const double *z,
                         const double *mass, const double *range2,
                         int nkernel, int precision,
                         double *ax, double *ay, double *az, double *pot,
                         double *W_per_set);

/* ---------------------------------------------- device-resident sweeps --- */
/* Add a seeded Gaussian displacement of standard deviation sigma to the n
 * device positions.  The draw for call c of particle p depends only on
 * (seed, c, p); c is a device-side counter that this kernel increments, so
 * repeated replays of a captured graph draw fresh kicks. */
int sphgrav_kick_positions_device(sphgrav_ctx *ctx, int n, double *x, double *y,
                                  double *z, double sigma, unsigned long long seed);
/* Reset the kick call counter to c (device-side, asynchronous). */
int sphgrav_kick_reset(sphgrav_ctx *ctx, unsigned long long c);

/* Capture the context's work between begin and end into a CUDA graph.
 * Inside the capture only *_device entry points may be called, and each of
 * them must have been called once before with the same sizes, so that every
 * buffer already exists.  The graph bakes in the context's work plan and
 * buffer addresses, and the settings in force (FP64 band, refine threshold,
 * error-scale keeping, theta): after any later call on the context that
 * changes them (other sizes, precision or variant, or a new value of one of
 * those settings) or after sphgrav_destroy,
 * sphgrav_graph_launch refuses with SPHGRAV_ERR_PROTOCOL and the graph must
 * be captured again.  Calls with the captured sizes may interleave with
 * replays. */
int sphgrav_capture_begin(sphgrav_ctx *ctx);
int sphgrav_capture_end(sphgrav_ctx *ctx, sphgrav_graph **graph);
int sphgrav_graph_launch(sphgrav_graph *graph, int repeats);
/* 1 while the graph may be replayed (see above), else 0. */
int sphgrav_graph_valid(const sphgrav_graph *graph);
/* Releases a graph.  Called while this thread captures (a garbage-collected
 * handle, say), the release waits until the capture ends: destroying a CUDA
 * graph is not allowed during a capture and would invalidate it. */
int sphgrav_graph_destroy(sphgrav_graph *graph);

/* ------------------------------------------------------------ tuning --- */
/* Time the kernel variants on the sets described by (nsets, offsets) with the
 * given device data and keep the fastest per (precision, N bucket).  Later
 * calls in that bucket use it. */
int sphgrav_autotune(sphgrav_ctx *ctx, int nsets, const int *offsets,
                     const double *x, const double *y, const double *z,
                     const double *mass, const double *range2,
                     int nkernel, int precision);
/* Persist / restore the tuning table (a small JSON file). */
int sphgrav_tuning_save(sphgrav_ctx *ctx, const char *path);
int sphgrav_tuning_load(sphgrav_ctx *ctx, const char *path);
/* Split-FP32 only: pairs with r < factor * max(H_i, H_j) are evaluated in
 * FP64 (default 1.0 = only the softened near field, r < max H).  A wider
 * band lowers the error of particles whose acceleration cancels and costs
 * time in proportion to the pairs it moves (~factor^3 times the near-field
 * pairs).  Factor in [1, 16].  No reference counterpart. */
int sphgrav_set_fp64_band(sphgrav_ctx *ctx, double factor);
/* Split-FP32 only: FP64 refine of ill-conditioned rows.  The split-FP32
 * kernel keeps, per row, G = sqrt(sum over its 256-source j-tiles of
 * |FP32 tile sum of the acceleration|^2), the scale of its FP32 rounding
 * error.  Rows with G > threshold * |a| -- particles whose acceleration
 * cancels, e.g. near a star's centre or between two stars -- are recomputed
 * in FP64 on the device in the same call (no host round trip; capturable),
 * so their relative error is that of the FP64 kernel.  Rows lying more than
 * 8 H from the centre of their row tile (where the FP32 rounding of their
 * tile-relative position shifts them measurably) are recomputed too.
 * Default 1.0 (0.1-0.4% of the rows of the benchmark workloads); 0 turns the
 * refine off.  No reference counterpart. */
int sphgrav_set_refine(sphgrav_ctx *ctx, double threshold);
/* Rows the last split-FP32 call recomputed in FP64 (0 when the refine was
 * off or the call was not split-FP32).  Synchronises the context's stream. */
int sphgrav_last_refine_rows(sphgrav_ctx *ctx, long long *rows);
/* Keep (on != 0) the per-row error scale G of later split-FP32 calls, and
 * copy the last call's G (caller order, n = all particles of the call) to
 * host memory; rows far from their tile centre read +infinity.
 * sphgrav_error_scale returns SPHGRAV_ERR_PROTOCOL when the last call kept
 * no scale of n rows.  Diagnostics; no reference counterpart. */
int sphgrav_keep_error_scale(sphgrav_ctx *ctx, int on);
int sphgrav_error_scale(sphgrav_ctx *ctx, int n, double *G);
/* SPHGRAV_TREE: opening angle theta in [0, 2] (default 0.3, the value
 * main.f:269 passes to gpu_init_dev_).  A node is opened when the gap
 * between its box and the walking group's box is at most l / theta (l its
 * edge length) or at most the largest H of either; theta = 0 opens every
 * node and gives the direct sum. */
int sphgrav_set_theta(sphgrav_ctx *ctx, double theta);
/* SPHGRAV_TREE: walking groups of the last tree call and how many of them
 * were handed to the direct FP64 sum (groups with more than 8,192 particles
 * within the largest H of their box; their rows are exact direct sums).
 * Both are -1 after a captured call (its counts stay on the device).
 * Either pointer may be NULL. */
int sphgrav_tree_stats(sphgrav_ctx *ctx, int *groups, int *heavy);
/* Force a kernel variant by index (-1 = automatic) for a precision. */
int sphgrav_force_variant(sphgrav_ctx *ctx, int precision, int variant);
/* Number of kernel variants and a printable name of each. */
int sphgrav_variant_count(int precision);
const char *sphgrav_variant_name(int precision, int variant);

/* ----------------------------------------------- no device allocation ---
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (during a CUDA graph capture, under a host's own memory pool, or
 * after start-up): FP64 forces of one set, all pointers DEVICE pointers of
 * length n, every row computed, enqueued on `stream` (a cudaStream_t; NULL is
 * the default stream).  Calls no cudaMalloc/cudaFree or allocating routine;
 * its only scratch is a static device array of SPHGRAV_NOALLOC_SCRATCH_BYTES
 * that every GPU loading this library holds until the process exits, which
 * caps n at SPHGRAV_NOALLOC_MAX_N (SPHGRAV_ERR_TOO_LARGE beyond).  The first
 * call on a device looks up that array's device address; make that first
 * call before any stream capture.  All calls share the array: calls that
 * overlap on the GPU (other streams, other host threads) race.  Particle data
 * are not validated (mass > 0 and range2 != 0 are the caller's contract). */
#define SPHGRAV_NOALLOC_SCRATCH_BYTES (8u << 20)
#define SPHGRAV_NOALLOC_MAX_N 262144
int sphgrav_forces_fp64_noalloc(int n, const double *x, const double *y, const double *z,
                                const double *mass, const double *range2, int nkernel,
                                double *ax, double *ay, double *az, double *pot,
                                void *stream);

/* ------------------------------------------------------- diagnostics --- */
const char *sphgrav_status_string(int status);
/* Last error message recorded on this thread (CUDA error text and context). */
const char *sphgrav_last_error_message(void);
/* Kernels launched by this library since the process started. */
unsigned long long sphgrav_launch_count(void);
/* Work items and j-chunks of the last computation (for tests and tuning). */
int sphgrav_last_plan_info(sphgrav_ctx *ctx, int *nitems, int *nchunks_max,
                           int *variant);
/* The work plan a call on whole sets would use, computed on the host only
 * (no context, no GPU needed): `resident` persistent CTAs of `variant` of
 * `precision`.  Writes the item and partial-slot counts and, for up to `cap`
 * items in queue order, 6 ints each: set, row tile, chunk, slot, first and
 * end source slot of the chunk (set-local).  For tests and tuning; no
 * counterpart in the reference. */
int sphgrav_plan_preview(int nsets, const int *offsets, int precision, int variant, int resident,
                         int *nitems, int *nslots, int *items, int cap);
/* Kernel timing: while enabled, CUDA events are recorded on the context's
 * stream around every pair-sum kernel launch (not inside graph captures);
 * sphgrav_profile_read returns the summed kernel milliseconds and launch
 * count since the previous read (it synchronises the stream). */
int sphgrav_profile_enable(sphgrav_ctx *ctx, int on);
int sphgrav_profile_read(sphgrav_ctx *ctx, double *kernel_ms, int *launches);
/* Phase accounting of the split-FP32 pair kernel, a diagnostic build
 * (`python -m starsmasher_b200.build --phases` compiles the kernel with
 * -DSG_PHASES into libsphgrav_b200_phases.so; the default library returns
 * SPHGRAV_ERR_UNSUPPORTED).  While sphgrav_profile_enable is on, every
 * split-FP32 launch adds the SM cycles its warps spend per phase; this call
 * synchronises the stream, copies the 16 counters and zeroes them.  Order:
 * consumer item fetch + barrier, row loads, waits for a staged tile, far loop,
 * checked loop, FP64 near pairs, item end; producer waits, producer work;
 * then counts of far and checked (warp, tile) pairs, near_eval calls and
 * items per consumer warp.  No counterpart in the reference. */
int sphgrav_phase_read(sphgrav_ctx *ctx, unsigned long long *counters, int n);
/* FP32 FMA throughput probe: runs a packed-FMA loop for about `iters`
 * iterations per thread on the context's device and returns the measured
 * TFLOP/s (2 flops per FMA) in *tflops. */
int sphgrav_fp32_peak_probe(sphgrav_ctx *ctx, int iters, double *tflops);
/* Self-test of the device-side failure path: a one-warp kernel waits, with
 * the pair kernels' bounded mbarrier poll, on a barrier that nothing arrives
 * on, gives up after `polls` polls (1..65536) and sets the context's device
 * error flag as a timed-out pair kernel does.  Returns
 * SPHGRAV_ERR_DEVICE_TIMEOUT (expected) after clearing the flag; the
 * context stays usable.  Blocking. */
int sphgrav_selftest_wait_timeout(sphgrav_ctx *ctx, int polls);
/* FP64 FMA throughput probe: eight independent DFMA chains per thread for
 * `iters` iterations; the measured TFLOP/s (2 flops per FMA) in *tflops. */
int sphgrav_fp64_peak_probe(sphgrav_ctx *ctx, int iters, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* SPHGRAV_B200_H */
