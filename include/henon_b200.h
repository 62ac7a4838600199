/*
 * henon_b200.h -- C ABI of the B200-native Henon-map tracking library
 * (libhenon_b200.so).
 *
 * Every entry point takes plain pointers and sizes, returns an hm_status and
 * never exits the process.  The message of the last failure on the calling
 * thread is available from hm_last_error().
 *
 * Reference interfaces replaced (paths inside carlidel/henon_map_cpp):
 *   - src/bind.cpp:224-577      pybind11 module `henon_map_engine`
 *   - src/henon.h:41-447        particles_4d[_gpu], henon_tracker[_gpu], the
 *                               tangent-map, indicator and storage classes
 *   - src/modulation.h:12-22    modulation tables
 *   - src/dynamic_indicator.h   birkhoff_weights
 *
 * Device memory layout (HBM):
 *   particles : structure of arrays, double x[n], px[n], y[n], py[n],
 *               uint32 steps[n], uint8 valid[n], uint8 ghost[n],
 *               uint64 idx[n], idx_base[n]   (n includes ghost particles)
 *   tracker   : one 32-byte record per turn {sin wx, cos wx, sin wy, cos wy}
 *               so that a chunk of turns is one contiguous bulk copy.
 *   matrices  : double[n][16] row-major 4x4 per particle (as the reference).
 *   vectors   : double[n][4].
 */
#ifndef HENON_B200_H
#define HENON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hm_status {
    HM_OK = 0,
    HM_ERR_INVALID_ARG = 1,        /* bad size, pointer or option            */
    HM_ERR_BUDGET = 2,             /* "The number of turns is too large."    */
    HM_ERR_CUDA = 3,               /* a CUDA runtime call failed             */
    HM_ERR_TIMEOUT = 4,            /* a bounded device wait gave up          */
    HM_ERR_CANCELLED = 5,          /* the cancel callback asked to stop      */
    HM_ERR_OOM = 6,                /* device allocation failed               */
    HM_ERR_UNKNOWN_MODULATION = 7, /* "Unknown modulation kind"              */
    HM_ERR_NOT_SUPPORTED = 8,      /* option not provided by this build      */
    HM_ERR_NO_DEVICE = 9           /* no CUDA device visible                 */
} hm_status;

/* Arithmetic of the map kernels.
 * HM_ARITH_EXACT: every multiply and add is a separately rounded IEEE-754
 *   binary64 operation in the reference's operation order (no contraction to
 *   FMA) -- results are bit-identical to the reference CPU path and to the
 *   reference CUDA path built with --fmad=false.
 * HM_ARITH_FAST: fused multiply-adds and reassociated polynomials; agrees
 *   with EXACT to rounding error per turn. */
typedef enum hm_arith { HM_ARITH_EXACT = 0, HM_ARITH_FAST = 1 } hm_arith;

/* Particle fields for hm_particles_get (host copies, like the reference's
 * getters, src/henon.cu:1444-1482, 1646-1676). */
typedef enum hm_field {
    HM_FIELD_X = 0,        /* double  */
    HM_FIELD_PX = 1,       /* double  */
    HM_FIELD_Y = 2,        /* double  */
    HM_FIELD_PY = 3,       /* double  */
    HM_FIELD_STEPS = 4,    /* uint32  */
    HM_FIELD_VALID = 5,    /* uint8   */
    HM_FIELD_GHOST = 6,    /* uint8   */
    HM_FIELD_IDX = 7,      /* uint64  */
    HM_FIELD_IDX_BASE = 8  /* uint64  */
} hm_field;

/* Elementwise observables (src/henon.cu:67-111 and 979-1121). */
typedef enum hm_observable {
    HM_OBS_RADIUS = 0,     /* sqrt(x^2+px^2+y^2+py^2) */
    HM_OBS_ACTION = 1,     /* x^2+px^2+y^2+py^2        */
    HM_OBS_ACTION_X = 2,   /* x^2+px^2                 */
    HM_OBS_ACTION_Y = 3,   /* y^2+py^2                 */
    HM_OBS_ANGLE_X = 4,    /* atan2(px, x)             */
    HM_OBS_ANGLE_Y = 5     /* atan2(py, y)             */
} hm_observable;

typedef struct hm_particles hm_particles;
typedef struct hm_tracker hm_tracker;

/* ---- library ----------------------------------------------------------- */

/* Message of the last failure on this thread ("" if none). */
const char *hm_last_error(void);
/* ABI version of this library (major * 10000 + minor * 100 + patch). */
int hm_version(void);
/* Number of CUDA devices visible (0 when none); never fails. */
int hm_device_count(void);

/* Called between turn chunks of every long operation; a non-zero return
 * stops the operation with HM_ERR_CANCELLED after the state has been made
 * consistent (replaces check_keyboard_interrupt, src/henon.cu:7-15). */
typedef int (*hm_cancel_fn)(void *ctx);
hm_status hm_set_cancel_callback(hm_cancel_fn fn, void *ctx);

/* Launch shape of the chunked tracking kernels: threads per block (32..256,
 * multiple of 32), particles per thread (1, 2 or 4), turns of the first
 * chunk and the cap of the doubling chunk length.  Process-wide; chosen by
 * the autotuner.  Results do not depend on it. */
hm_status hm_set_track_config(int threads, int per_thread, uint32_t chunk0,
                              uint32_t chunk_max);
hm_status hm_get_track_config(int *threads, int *per_thread,
                              uint32_t *chunk0, uint32_t *chunk_max);
/* How the tracking kernels read the per-turn records {sin wx, cos wx,
 * sin wy, cos wy}: 0 = straight from global memory (a broadcast load per
 * warp and turn); otherwise one thread per block brings stage_turns turns
 * of records at a time into shared memory with a bulk copy (TMA,
 * double-buffered, bounded waits) and every warp reads them from there.
 * stage_turns is 0 or a power of two in [16, 512] (default 256); runs of
 * one chunk use direct reads.  Process-wide; results do not depend on it.
 * A staged copy that does not land within its bounded wait makes the call
 * return HM_ERR_TIMEOUT.  After HM_ERR_TIMEOUT the particles' coordinates
 * and steps are unspecified (the chunk that gave up may have moved some of
 * them, and its survivors may still be in the scratch lists), and
 * global_steps is left unchanged: reset the particles before reusing them. */
hm_status hm_set_track_staging(uint32_t stage_turns);
hm_status hm_get_track_staging(uint32_t *stage_turns);

/* ---- host numerics ----------------------------------------------------- */

/* omega(n) for n in [offset, offset+n_turns) for both planes.
 * kind: "sps", "basic", "none", "gaussian", "uniform"
 * (pick_a_modulation, src/modulation.cpp:101-134; "none" fills the constant
 * omega, see the library documentation). */
hm_status hm_modulation(const char *kind, uint32_t n_turns, double omega_x,
                        double omega_y, double omega_0, double epsilon,
                        uint32_t offset, double *omega_x_out,
                        double *omega_y_out);
/* sps_modulation, src/modulation.cpp:31-60 (start < end). */
hm_status hm_sps_modulation(double tune, double epsilon, int32_t start,
                            int32_t end, double *out);
/* basic_modulation, src/modulation.cpp:3-11 (start < end). */
hm_status hm_basic_modulation(double tune, double omega, double epsilon,
                              int32_t start, int32_t end, double *out);
/* birkhoff_weights, src/dynamic_indicator.cpp:63-79. */
hm_status hm_birkhoff_weights(uint32_t n_weights, double *out);

/* ---- tracker (henon_tracker_gpu, src/henon.cu:3114-3185) --------------- */

hm_status hm_tracker_create(uint32_t n_turns, double omega_x, double omega_y,
                            const char *modulation_kind, double omega_0,
                            double epsilon, uint32_t offset, hm_tracker **out);
/* henon_tracker_gpu::compute_a_modulation, src/henon.cu:3135-3153. */
hm_status hm_tracker_compute_a_modulation(hm_tracker *t, uint32_t n_turns,
                                          double omega_x, double omega_y,
                                          const char *modulation_kind,
                                          double omega_0, double epsilon,
                                          uint32_t offset);
hm_status hm_tracker_destroy(hm_tracker *t);
/* Turns the tables hold (allowed_steps in the reference). */
hm_status hm_tracker_allowed_steps(const hm_tracker *t, uint64_t *out);
/* Host copies of the four tables, each of allowed_steps doubles. */
hm_status hm_tracker_get_tables(const hm_tracker *t, double *sin_x,
                                double *cos_x, double *sin_y, double *cos_y);
/* Device pointer to the interleaved {sx,cx,sy,cy} turn records. */
hm_status hm_tracker_device_tables(const hm_tracker *t, const double **out);
hm_status hm_tracker_set_arith(hm_tracker *t, hm_arith arith);
hm_status hm_tracker_get_arith(const hm_tracker *t, hm_arith *out);

/* ---- particles (particles_4d_gpu, src/henon.cu:1154-1691) -------------- */

hm_status hm_particles_create(const double *x, const double *px,
                              const double *y, const double *py, size_t n,
                              hm_particles **out);
hm_status hm_particles_destroy(hm_particles *p);
/* particles_4d::reset, src/henon.cu:727-735 (global_steps is kept). */
hm_status hm_particles_reset(hm_particles *p);
/* Total size including ghosts, base particle count, ghosts per particle. */
hm_status hm_particles_size(const hm_particles *p, size_t *n_total,
                            size_t *n_particles, size_t *n_ghosts);
hm_status hm_particles_global_steps(const hm_particles *p, uint32_t *out);
/* Host copy of one field (n_total elements of the field's type). */
hm_status hm_particles_get(const hm_particles *p, hm_field field,
                           void *host_out);
/* Device pointer of one field (valid until the next add_ghost/destroy). */
hm_status hm_particles_device_ptr(const hm_particles *p, hm_field field,
                                  void **out);
/* Elementwise observable of all n_total entries (GPU getters). */
hm_status hm_particles_observable(const hm_particles *p, hm_observable kind,
                                  double *host_out);

/* Ghost particles (particles_4d::add_ghost, src/henon.cu:737-818): one ghost
 * per base particle, displaced by `module` along "x", "px", "y", "py" or an
 * isotropic "random" direction (the set's default-seeded mt19937_64, as the
 * reference).  Like the reference's GPU class (:1247-1255) the device state
 * is rebuilt from the initial conditions. */
hm_status hm_particles_add_ghost(hm_particles *p, double module,
                                 const char *direction);
/* renormalize (src/henon.cu:1257-1282). */
hm_status hm_particles_renormalize(hm_particles *p, double module);
/* get_displacement_module (:1284-1343): double[n_particles][n_ghosts]. */
hm_status hm_particles_displacement_module(const hm_particles *p,
                                           double *host_out);
/* get_displacement_direction (:1345-1442): double[4][n_particles][n_ghosts]. */
hm_status hm_particles_displacement_direction(const hm_particles *p,
                                              double *host_out);
/* The displacement (ghost) Lyapunov loop of the reference's notebooks
 * (tests/test_new_standard.ipynb:477-479), which a Python caller runs as
 *     for step in range(n_steps):
 *         tracker.track(p, every, mu, barrier)
 *         lyap += log(p.get_displacement_module() / module)
 *         p.renormalize(module)
 * over add_ghost / renormalize / get_displacement_module (src/henon.cu:
 * 737-818, 1257-1343), in fused launches: each thread carries a base
 * particle and its ghosts in registers.  Coordinates, steps and
 * global_steps end as after that loop, bit for bit; host_out
 * (double[n_particles][n_ghosts]) receives the sums of log(d / module)
 * over this call's steps (CUDA's log: each term within an ulp of the host
 * loop's).  1 to 4 ghosts per particle (HM_ERR_NOT_SUPPORTED beyond).  No
 * kicks.  Synchronous; cancellable between launches. */
hm_status hm_track_ghost_lyapunov(hm_tracker *t, hm_particles *p,
                                  uint32_t n_steps, uint32_t every, double mu,
                                  double barrier, double module,
                                  double *host_out);
/* henon_tracker_gpu::get_tangent_matrix (src/henon.cu:3187-3219), computed
 * on the host like the reference: double[n_total][16]. */
hm_status hm_tracker_tangent_matrices(const hm_tracker *t,
                                      const hm_particles *p, double mu,
                                      int reverse, double *host_out);

/* ---- tracking ---------------------------------------------------------- */

/* henon_tracker_gpu::track, src/henon.cu:3155-3185: n_turns turns of the
 * map on every particle, fused into chunked multi-turn launches.
 * kick_module not NaN: every turn first kicks each particle by kick_module
 * along a random direction (random_4d_kick, src/henon.cu:387-405).  Unlike
 * the reference's clock()-seeded stream, the direction is a function of
 * (the particles' kick seed, particle index, table index of the turn):
 * Philox4x32-10 and Marsaglia's uniform point on the 3-sphere, so a run is
 * reproducible and independent of launch shape and chunking.  Backward
 * turns subtract the kick of the same table index after the inverse
 * sextupole, undoing the forward turn's kick. */
hm_status hm_track(hm_tracker *t, hm_particles *p, uint32_t n_turns,
                   double mu, double barrier, double kick_module, int inverse);
/* Key of the kicks of hm_track for these particles (0 after creation). */
hm_status hm_particles_set_kick_seed(hm_particles *p, uint64_t seed);
hm_status hm_particles_get_kick_seed(const hm_particles *p, uint64_t *seed);

/* Kernel-level form of the same operation on caller-owned device arrays
 * (the loop body of gpu_henon_track, src/henon.cu:636-691).  start_step is
 * the steps value shared by all live particles; tables holds table_len
 * records.  workspace must hold hm_track_workspace_bytes(n) bytes of device
 * memory (NULL is allowed when n_turns fits one chunk).  stream is a
 * cudaStream_t (NULL = legacy default stream).  Synchronous. */
size_t hm_track_workspace_bytes(size_t n);
hm_status hm_track_device(double *x, double *px, double *y, double *py,
                          uint32_t *steps, size_t n, const double *tables,
                          uint64_t table_len, uint32_t start_step,
                          uint32_t n_turns, double mu, double barrier,
                          int inverse, hm_arith arith, void *workspace,
                          void *stream);

/* ---- tangent map (matrix_4d_vector_gpu, vector_4d_gpu) ------------------
 * One 4x4 matrix / 4-vector per particle on the device.  Each call is one
 * elementwise launch with the reference's arithmetic order, so results are
 * bit-identical to the reference CUDA build with --fmad=false. */

typedef struct hm_matrices hm_matrices;
typedef struct hm_vectors hm_vectors;

/* matrix_4d_vector_gpu(N): N identity matrices (src/henon.cu:1789-1808). */
hm_status hm_matrices_create(size_t n, hm_matrices **out);
hm_status hm_matrices_destroy(hm_matrices *m);
hm_status hm_matrices_size(const hm_matrices *m, size_t *n);
/* Back to identity (the reference's reset is a no-op, src/henon.cu:1815). */
hm_status hm_matrices_reset(hm_matrices *m);
/* M <- DF(x; table[global_steps]) * M (structured_multiply, :1827-1835). */
hm_status hm_matrices_structured_multiply(hm_matrices *m, const hm_tracker *t,
                                          const hm_particles *p, double mu);
/* M <- DF(x; table[global_steps]) (set_with_tracker, :1837-1845). */
hm_status hm_matrices_set_with_tracker(hm_matrices *m, const hm_tracker *t,
                                       const hm_particles *p, double mu);
/* explicit_copy (:1907-1912). */
hm_status hm_matrices_copy(hm_matrices *dst, const hm_matrices *src);
/* Host copy, double[n][16] row-major (get_matrix, :1914-1946). */
hm_status hm_matrices_get(const hm_matrices *m, double *host_out);
/* out[i] = M[i] rv[i], double[n][4] (get_vector, :1847-1905). */
hm_status hm_matrices_get_vector(const hm_matrices *m, const double *host_rv,
                                 double *host_out);

/* vector_4d_gpu(rv): double[n][4] (src/henon.cu:1948-1971). */
hm_status hm_vectors_create(const double *host, size_t n, hm_vectors **out);
hm_status hm_vectors_destroy(hm_vectors *v);
/* set_vectors (:1978-2007): host double[n][4], or one 4-vector repeated
 * when broadcast != 0. */
hm_status hm_vectors_set(hm_vectors *v, const double *host, int broadcast);
/* v <- M v (multiply, :2009-2013). */
hm_status hm_vectors_multiply(hm_vectors *v, const hm_matrices *m);
/* v <- v / |v| (normalize, :2015-2019). */
hm_status hm_vectors_normalize(hm_vectors *v);
hm_status hm_vectors_get(const hm_vectors *v, double *host_out);

/* ---- indicator constructs ------------------------------------------------ */

typedef struct hm_lyapunov hm_lyapunov;
typedef struct hm_megno hm_megno;
typedef struct hm_megno_birkhoff hm_megno_birkhoff;
typedef struct hm_tune_birkhoff hm_tune_birkhoff;
typedef struct hm_storage hm_storage;

/* lyapunov_birkhoff_construct (one window, src/henon.cu:2042-2128) and
 * lyapunov_birkhoff_construct_multi (src/henon.cu:2130-2220): per add, for
 * every window w with idx < n_w: raw_w += log|v|/n_w, b_w += log|v| w[idx].
 * (The reference's one-window add has no idx < n_w guard, :2103; here it
 * has.) */
hm_status hm_lyapunov_create(size_t n, const uint64_t *n_weights,
                             size_t n_windows, hm_lyapunov **out);
hm_status hm_lyapunov_destroy(hm_lyapunov *h);
hm_status hm_lyapunov_reset(hm_lyapunov *h);
hm_status hm_lyapunov_change_weights(hm_lyapunov *h, uint64_t n_weights);
hm_status hm_lyapunov_add(hm_lyapunov *h, const hm_vectors *v);
hm_status hm_lyapunov_windows(const hm_lyapunov *h, size_t *n_windows);
hm_status hm_lyapunov_get_weights(const hm_lyapunov *h, size_t window,
                                  double *host_out);
/* birkhoff 0: get_values_raw, 1: get_values_b; double[n_windows][n]. */
hm_status hm_lyapunov_get(const hm_lyapunov *h, int birkhoff,
                          double *host_out);

/* megno_construct (src/henon.cu:2223-2299): with a = |A|_F, b = |B|_F,
 * L1 += log10(a/b)*idx, L2 += L1/idx, value = L2/idx (idx from 1). */
hm_status hm_megno_create(size_t n, hm_megno **out);
hm_status hm_megno_destroy(hm_megno *h);
hm_status hm_megno_reset(hm_megno *h);
hm_status hm_megno_add(hm_megno *h, const hm_matrices *a, const hm_matrices *b);
hm_status hm_megno_get(const hm_megno *h, double *host_out);

/* megno_birkhoff_construct (src/henon.cu:2302-2426): windows T_j,
 * L2_j += L1 * w_Tj[idx-1] / idx while idx <= T_j; double[n_samples][n]. */
hm_status hm_megno_birkhoff_create(size_t n, const uint64_t *turn_samples,
                                   size_t n_samples, hm_megno_birkhoff **out);
hm_status hm_megno_birkhoff_destroy(hm_megno_birkhoff *h);
hm_status hm_megno_birkhoff_reset(hm_megno_birkhoff *h);
hm_status hm_megno_birkhoff_add(hm_megno_birkhoff *h, const hm_matrices *a,
                                const hm_matrices *b);
hm_status hm_megno_birkhoff_get(const hm_megno_birkhoff *h, double *host_out);

/* tune_birkhoff_construct (src/henon.cu:2428-2655): phase advance
 * atan2(p, q) wrapped to (0, 2pi], weighted into [0, T) and [T, 2T).
 * which: 0 tune1_x, 1 tune1_y, 2 tune2_x, 3 tune2_y; double[n_samples][n].
 * Accumulators start at zero (the reference leaves them uninitialised
 * until reset()). */
hm_status hm_tune_birkhoff_create(size_t n, const uint64_t *turn_samples,
                                  size_t n_samples, hm_tune_birkhoff **out);
hm_status hm_tune_birkhoff_destroy(hm_tune_birkhoff *h);
hm_status hm_tune_birkhoff_reset(hm_tune_birkhoff *h);
hm_status hm_tune_birkhoff_first_add(hm_tune_birkhoff *h, const hm_particles *p);
hm_status hm_tune_birkhoff_add(hm_tune_birkhoff *h, const hm_particles *p);
hm_status hm_tune_birkhoff_get(const hm_tune_birkhoff *h, int which,
                               double *host_out);

/* storage_4d_gpu (src/henon.cu:3351-3462): batch snapshots of x, px, y, py;
 * double[batch][n] per field.  store() past batch_size is refused (the
 * reference writes past its buffers). */
hm_status hm_storage_create(size_t n, size_t batch, hm_storage **out);
hm_status hm_storage_destroy(hm_storage *h);
hm_status hm_storage_store(hm_storage *h, const hm_particles *p);
hm_status hm_storage_reset(hm_storage *h);
hm_status hm_storage_size(const hm_storage *h, size_t *n, size_t *batch,
                          size_t *stored);
hm_status hm_storage_get(const hm_storage *h, hm_field field, double *host_out);
hm_status hm_storage_device_ptr(const hm_storage *h, hm_field field,
                                const double **out);

/* ---- fused tracking + indicators ----------------------------------------
 * hm_track_indicators runs n_turns iterations of the per-turn loop that the
 * reference drives from Python (tests/test_construct.ipynb,
 * tests/test_new_standard.ipynb), in chunked multi-turn launches:
 *     matrix_old <- matrix                     (when given)
 *     track(p, 1, mu, barrier)                 (hm_track)
 *     matrix.structured_multiply(t, p, mu)     (when matrix)
 *     megno.add(matrix, matrix_old)            (when megno)
 *     megno_birkhoff.add(matrix, matrix_old)   (when megno_birkhoff)
 *     J.set_with_tracker(t, p, mu); vectors.multiply(J);
 *     lyapunov.add(vectors); vectors.normalize()  (when vectors)
 *     tune.add(p)                              (when tune)
 * Every handle ends in the state the loop leaves it in, bit for bit.  The
 * MEGNO layer-3 value is also recorded into megno_samples_out[j][i] when
 * megno's add counter equals megno_sample_turns[j].  All construct sizes
 * must equal the particle count; the tracker needs global_steps + n_turns
 * + 1 table entries when a tangent part is on (structured_multiply reads
 * table[global_steps] after the turn). */
typedef struct hm_indicator_set {
    hm_matrices *matrix;
    hm_matrices *matrix_old;
    hm_megno *megno;
    hm_megno_birkhoff *megno_birkhoff;
    hm_vectors *vectors;
    hm_lyapunov *lyapunov;
    hm_tune_birkhoff *tune;
    const uint64_t *megno_sample_turns;
    size_t n_megno_samples;
    double *megno_samples_out; /* host double[n_megno_samples][n] or NULL */
    /* 0: the loop above (DF of the new point with table[global_steps], as
     * structured_multiply after track); 1: DF of the turn itself, at the
     * point before the turn with table[steps] (the tangent map of the
     * orbit; needs no extra table entry). */
    int jacobian_of_turn;
} hm_indicator_set;

hm_status hm_track_indicators(hm_tracker *t, hm_particles *p, uint32_t n_turns,
                              double mu, double barrier,
                              const hm_indicator_set *set);
/* henon_tracker::megno (src/henon.cu:2755-2887) on the GPU: MEGNO of the
 * tangent map of the orbit (the Jacobian of each turn at the point before
 * it, accumulated as megno_construct does, src/henon.cu:2253-2284) at the
 * turn counts turn_samples, host_out double[n_total][n_samples].  As in the
 * reference the call tracks the particles n_turns turns, with kick_module
 * (NaN: none; hm_track's reproducible kicks) and inverse (backward turns,
 * each with the Jacobian of the backward turn, inverse_tangent_matrix
 * src/henon.cu:224-249; global_steps decreases). */
hm_status hm_tracker_megno(hm_tracker *t, hm_particles *p, uint32_t n_turns,
                           double mu, double barrier, double kick_module,
                           int inverse, const uint64_t *turn_samples,
                           size_t n_samples, double *host_out);

/* ---- batched heterogeneous tracking ---------------------------------------
 * Replaces the reference's one-process-per-parameter-set sweeps
 * (htcondor_jobs/compose_config.py:3-15, run_sim.py:41-74): many
 * (omega_x, omega_y, epsilon, mu, barrier) sets, each with its own particle
 * count and turn budget, tracked together.  Each set's particles are
 * advanced exactly as hm_track would advance them alone (bit-identical);
 * hm_batch_run replays the whole batch as one captured CUDA graph of
 * persistent chunk launches and planning kernels. */
typedef struct hm_batch hm_batch;
typedef struct hm_batch_set {
    double omega_x, omega_y;      /* tunes (henon_tracker arguments)        */
    const char *modulation_kind;  /* NULL means "sps"                       */
    double omega_0, epsilon;
    uint32_t offset;
    uint32_t n_turns;             /* turn budget of this set                */
    uint64_t n_particles;
    double mu;
    double barrier;
} hm_batch_set;

hm_status hm_batch_create(size_t n_sets, const hm_batch_set *sets,
                          hm_batch **out);
hm_status hm_batch_destroy(hm_batch *b);
/* Arithmetic, particles per thread (1, 2, 4) and the chunk schedule (first
 * chunk, cap of the doubling length; default 512 and 4096); chosen by the
 * autotuner. */
hm_status hm_batch_configure(hm_batch *b, hm_arith arith, int per_thread,
                             uint32_t chunk0, uint32_t chunk_max);
/* Splits the sets into `groups` (1..16) groups of about equal work, each
 * tracked by its own chain of chunk launches on its own stream, so that
 * one group's chunk ramp-down overlaps another group's work (default 16,
 * at most the number of sets).  Results do not depend on it. */
hm_status hm_batch_set_groups(hm_batch *b, int groups);
/* Grid of each group's chunk kernel: share x (the group's particles x
 * turns) / (all sets'), as a fraction of the device's resident blocks, at
 * most all of them (default 1.5; 0 gives every group the whole device).
 * Smaller grids running side by side spend less of each launch in its
 * last, partly empty round of tiles.  Results do not depend on it. */
hm_status hm_batch_set_grid_share(hm_batch *b, double share);
hm_status hm_batch_size(const hm_batch *b, uint64_t *n_total,
                        uint32_t *n_chunks);
/* Initial conditions of all sets, concatenated in set order (host). */
hm_status hm_batch_load(hm_batch *b, const double *x, const double *px,
                        const double *y, const double *py);
/* Tracks every set from its initial conditions to its budget.  use_graph:
 * capture once, replay after. Synchronous. */
hm_status hm_batch_run(hm_batch *b, int use_graph);
/* Host copy of x, px, y, py (double) or steps (uint32), concatenated. */
hm_status hm_batch_get(const hm_batch *b, hm_field field, void *host_out);

/* ---- tunes from turn-by-turn orbits ---------------------------------------
 * An orbit is n_samples snapshots of n particles per coordinate, laid out
 * [sample][particle] on the device (storage_4d_gpu's layout).  Windows are
 * inclusive sample ranges [from[j], to[j]]; the full orbit is appended as a
 * last window.  Output host double[n][2 (n_windows + 1)] = (tune_x,
 * tune_y) per window.
 *   method 0 -- Birkhoff tune (birkhoff_tune_vec, src/dynamic_indicator.cpp:
 *     198-253): 1 - sum w_i dtheta_i / 2pi, theta = atan2(p, q), dtheta
 *     wrapped by +2pi when negative, w = birkhoff_weights(to - from); NaN
 *     when a window holds a NaN; full orbit = samples [0, n_samples-1].
 *   method 1 -- FFT tune (fft_tune_vec, src/dynamic_indicator.cpp:255-330):
 *     Hann-windowed FFT of q + i p (cuFFT), interpolated peak, |1 - nu|;
 *     full orbit = samples [1, n_samples-1]. */
hm_status hm_orbit_tunes(const double *x, const double *px, const double *y,
                         const double *py, size_t n, size_t n_samples,
                         const uint32_t *from, const uint32_t *to,
                         size_t n_windows, int method, double *host_out);
/* The same on host arrays [n_samples][n] (storage_4d::tune_birkhoff /
 * tune_fft of the reference's host-side storage, src/henon.cu:3261-3329). */
hm_status hm_orbit_tunes_host(const double *x, const double *px, const double *y,
                              const double *py, size_t n, size_t n_samples,
                              const uint32_t *from, const uint32_t *to,
                              size_t n_windows, int method, double *host_out);
/* Tracks n_turns turns recording the orbit (sample 0 = the current state),
 * then Birkhoff tunes (and FFT tunes when fft_out is not NULL) of the
 * windows plus the full orbit, with each orbit's mean removed first when
 * remove_mean: henon_tracker::birkhoff_tunes (remove_mean 0) and
 * ::all_tunes (remove_mean 1), src/henon.cu:2890-3078.  kick_module (NaN:
 * none) and inverse are hm_track's: reproducible kicks keyed by the
 * particles' kick_seed, backward turns with global_steps decreasing.
 * Outputs host double[n_total][2 (n_windows + 1)].  Birkhoff sums are
 * added in segments of turns (within 1e-13 of the sequential sum). */
hm_status hm_tracker_orbit_tunes(hm_tracker *t, hm_particles *p, uint32_t n_turns,
                                 double mu, double barrier, double kick_module,
                                 int inverse, const uint32_t *from,
                                 const uint32_t *to, size_t n_windows,
                                 int remove_mean, double *birkhoff_out,
                                 double *fft_out);
/* Most particles hm_tracker_orbit_tunes records in one slice (0, the
 * default: as many as two thirds of the free device memory hold).  A cap
 * bounds the call's device memory; the FFT tunes and the orbit do not
 * depend on it, the Birkhoff sums only through their segments (1e-13).
 * Process-wide. */
hm_status hm_set_tune_slice_limit(size_t max_particles);
hm_status hm_get_tune_slice_limit(size_t *max_particles);
/* Tunes of a storage's snapshots (storage_4d::tune_birkhoff / tune_fft,
 * src/henon.cu:3261-3329). */
hm_status hm_storage_tunes(const hm_storage *s, const uint32_t *from,
                           const uint32_t *to, size_t n_windows, int method,
                           double *host_out);

/* ---- orbit-loss gradients (reverse-mode adjoint) ---------------------------
 * No counterpart in the reference (its tangent map is forward only,
 * src/henon.cu:175-313).  For every particle i of the device arrays x0..py0
 * the Birkhoff-weighted orbit loss
 *     L_i = sum_{k=0}^{n_turns-1} w_k (x^2+px^2+y^2+py^2)(after turn k),
 *     w = birkhoff_weights(n_turns),
 * is computed with the tracker's tables and arithmetic (the orbit is the
 * one hm_track follows); particles lost before n_turns get L_i = 0 and
 * survived[i] = 0.  mode 0 adds reverse-mode gradients: grad_ic[4][n] =
 * dL_i/d(x0, px0, y0, py0) and grad_theta[4][n] = dL_i/d(omega_x0,
 * omega_y0, epsilon, mu), omega_{x,y}0 = 2 pi tune_{x,y}, with checkpoints
 * every checkpoint_every turns and recomputation in between (workspace of
 * hm_adjoint_workspace_bytes).  mode 0 replays each segment from its
 * checkpoint into the workspace (the states are the forward orbit's, bit
 * for bit); mode 3 instead rebuilds them backwards with the map's exact
 * inverse from the state at the segment's end (no per-turn memory traffic;
 * reconstruction error bounded to one segment).  mode 1 gives grad_ic by
 * forward-mode tangent-map propagation (an independent J^T v) and, when
 * grad_theta is not NULL, grad_theta by forward propagation of the state's
 * derivatives with respect to theta alongside it; mode 2 the loss only.
 * Derivatives need an "sps" or "basic" modulation.  Synchronous. */
size_t hm_adjoint_workspace_bytes(size_t n, uint32_t n_turns,
                                  uint32_t checkpoint_every);
/* Particles per thread of mode 3's kernel (1 or 2).  Process-wide; chosen
 * by the autotuner; results do not depend on it. */
hm_status hm_set_adjoint_config(int per_thread);
hm_status hm_get_adjoint_config(int *per_thread);
hm_status hm_adjoint(const hm_tracker *t, const double *x0, const double *px0,
                     const double *y0, const double *py0, size_t n, double mu,
                     double barrier, uint32_t n_turns, uint32_t checkpoint_every,
                     int mode, double *loss, uint8_t *survived, uint32_t *steps,
                     double *grad_ic, double *grad_theta, void *workspace,
                     void *stream);

/* No counterpart in the reference.  The same operation as hm_track_device
 * for callers that cannot allocate device memory (an application that
 * reserves all device memory at start-up, a framework whose allocator owns
 * every device byte, a loop that cannot take cudaFree's device-wide
 * synchronisation): it calls no cudaMalloc, cudaFree or allocating library
 * routine.  Its scratch is a fixed device array built into the library
 * (room for HM_NOALLOC_MAX_PARTICLES particles, about 9 MiB, held by every
 * GPU that loads the library until the process exits); n above that limit
 * is rejected with HM_ERR_INVALID_ARG.  The first call on each device looks
 * up the array's device address (cudaGetSymbolAddress); that lookup can
 * load the library's device code onto the device, which takes device
 * memory (the array itself among it), so make that first call (n = 0
 * is enough) before the caller reserves its device memory and before any
 * stream capture.  The current device must own `stream` and the
 * arrays; a stream of another device is rejected with HM_ERR_INVALID_ARG.
 * All calls on a device share the array: calls that overlap on the GPU
 * race.  Particle state after HM_ERR_TIMEOUT is as for hm_track_device.
 * Synchronous. */
#define HM_NOALLOC_MAX_PARTICLES 131072u
hm_status hm_track_device_noalloc(double *x, double *px, double *y, double *py,
                                  uint32_t *steps, size_t n,
                                  const double *tables, uint64_t table_len,
                                  uint32_t start_step, uint32_t n_turns,
                                  double mu, double barrier, int inverse,
                                  hm_arith arith, void *stream);

/* ---- device memory ----------------------------------------------------- */

/* The library's device buffers (particles, tables, scratch) come from one
 * memory pool per device that keeps freed blocks for reuse, so a loop that
 * creates and destroys particle sets makes no allocation call into the
 * driver once the pool has grown.  This returns the pool's unused blocks
 * to the device (cf. torch.cuda.empty_cache); buffers in use are kept.
 * Waits for every device the library has allocated on. */
hm_status hm_release_cached_memory(void);

/* ---- measurement ------------------------------------------------------- */

/* Times every tracking kernel launch with CUDA events on its stream while
 * enabled (turning it on or off resets the totals). */
hm_status hm_set_profiling(int on);
/* Summed device time (ms) and number of timed tracking launches. */
hm_status hm_get_profile(double *kernel_ms, uint64_t *launches);
/* Work of the same timed launches: particles of their input lists and
 * their turns, each summed over the launches (the units of the roofline's
 * algorithmic bytes: 36 B in + 36 B out per list particle, 32 B of turn
 * records per turn). */
hm_status hm_get_profile_work(uint64_t *list_particles, uint64_t *chunk_turns);

/* FP64 FMA-chain microbenchmark on the current device: *tflops receives
 * the achieved FP64 rate (an FMA counts as 2 flops). */
hm_status hm_fp64_peak(double seconds_target, double *tflops, double *ms);

#ifdef __cplusplus
}
#endif

#endif /* HENON_B200_H */
