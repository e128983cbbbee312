/*
 * pybrown_b200 -- C ABI of the B200 (sm_100a) hydrodynamics library.
 *
 * Two tiers:
 *
 *  1. Reference ABI.  The exact symbols, signatures and argument meanings of
 *     pyBrown's native library libpyBrown (src/bdsim/clib/diff_tensor.c,
 *     src/bdsim/clib/bead.c), as bound by ctypes in src/bdsim/pyBrown/diffusion.py
 *     and src/bdsim/pyBrown/bead.py.  Host pointers, FP64, caller-owned
 *     buffers.  Each call copies its inputs to the GPU, runs the sm_100a
 *     kernels and copies the result back.  Like the reference these return
 *     void (check_overlaps returns its flag); a failure is reported on stderr
 *     and through pbg_last_error().
 *
 *  2. Device-resident API (pbg_*).  Device pointers, an explicit cudaStream_t,
 *     int status returns (PBG_OK or a negative PBG_ERR_* code).  A pbg_system
 *     handle owns the per-system tensors (D, B, Mff, Rff, R, positions) in HBM
 *     and advances Brownian / Stokesian dynamics without host round trips.
 *
 * No torch types appear here; Python binds this with ctypes.
 */
#ifndef PYBROWN_B200_H
#define PYBROWN_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PBG_API __attribute__((visibility("default")))
#else
#define PBG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define PBG_OK 0
#define PBG_ERR_CUDA -1       /* a CUDA runtime call failed */
#define PBG_ERR_ARG -2        /* invalid argument */
#define PBG_ERR_NOT_SPD -3    /* a Cholesky pivot was not positive */
#define PBG_ERR_ATTEMPTS -4   /* max_move_attempts exceeded (box.py:248,347) */
#define PBG_ERR_NOISE -5      /* the device noise pool ran out; step rolled back */
#define PBG_ERR_NOMEM -6      /* device allocation failed */
#define PBG_ERR_BARRIER -7    /* a bounded device-wide wait gave up */
#define PBG_ERR_NAN -8        /* a non-finite value was produced */
#define PBG_ERR_STATE -9      /* call out of order (e.g. step before set_state) */

/* Message of the last error recorded on the calling thread ("" if none). */
PBG_API const char *pbg_last_error(void);
/* ABI version: major * 10000 + minor * 100 + patch. */
PBG_API int pbg_version(void);
/* Number of kernels this library has launched in the process so far. */
PBG_API long long pbg_launch_count(void);
/* Launch calls the host has made (each kernel launched directly and each CUDA
 * graph launch count one; the kernels inside a graph do not). */
PBG_API long long pbg_host_launch_count(void);

/* ============================================================= Tier 1 ==== */
/* Reference ABI, drop-in replacements for libpyBrown's exports.            */

/* diff_tensor.c:73 -- free-space RPY mobility; caller passes a zeroed 9N^2 M. */
PBG_API void RPY_M_matrix(double *as, double *pointers, int number_of_beads, double *M_matrix);

/* diff_tensor.c:170 -- RPY mobility under Smith's Ewald summation. */
PBG_API void RPY_Smith_M_matrix(double *as, double *pointers, double box_length, double alpha,
                        int m_max, int n_max, int number_of_beads, double *M_matrix);

/* diff_tensor.c:270 -- Jeffrey-Onishi two-body resistance, 18 components. */
PBG_API void JO_2B_R_matrix(double ai, double aj, double rx, double ry, double rz, double *R_matrix);

/* diff_tensor.c:346 -- lubrication correction, accumulated (+=) into a 9N^2 buffer. */
PBG_API void JO_R_lubrication_correction_matrix(double *as, double *pointers, int number_of_beads,
                                        double cutoff_distance, int cichocki_correction,
                                        double *correction_matrix);

/* bead.c:27 -- minimum-image pair vectors, N x N x 3. */
PBG_API void pointer_pbc_matrix(double *positions, int number_of_beads, double box_length, double *pointers);

/* bead.c:99 -- mobile/immobile pair vectors, N_mob x N_immob x 3. */
PBG_API void pointer_immobile_pbc_matrix(double *positions_mobile, double *positions_immobile,
                                 int number_of_mobile, int number_of_immobile,
                                 double box_length, double *pointers);

/* bead.c:169 -- 1 if any non-bonded pair overlaps, else 0. */
PBG_API int check_overlaps(double *positions, double *as, int number_of_beads, double box_length,
                   double overlap_treshold, int *connection_matrix);

/* ============================================================= Tier 2 ==== */

/* ---- stateless device kernels (device pointers, stream-ordered) -------- */
/* Matrices are row-major with leading dimension ld (elements).  Results are
 * multiplied by `scale` on store, which is how the callers fold in the
 * kBT*1e19/eta (D) or 1e19/eta (Mff) factors of box.py:498-522. */

/* Pair vectors (bead.c:27-95) from device positions: rij is N*N*3. */
PBG_API int pbg_dev_pointer_matrix(const double *pos, int n_beads, double box_length, double *rij,
                           void *stream);

/* Free-space RPY (diff_tensor.c:73-166) from positions, minimum image in L. */
PBG_API int pbg_dev_rpy_matrix(const double *pos, const double *radii, int n_beads, double box_length,
                       double scale, double *M, int ld, void *stream);

/* Smith-Ewald RPY (diff_tensor.c:170-266) from positions. precision:
 * PBG_PREC_FP64 writes doubles to M; PBG_PREC_MIXED writes floats (M is a
 * float*).  Scratch (phase tables) is taken from the stream-ordered pool. */
PBG_API int pbg_dev_smith_matrix(const double *pos, const double *radii, int n_beads, double box_length,
                         double alpha, int m_max, int n_max, double scale, int precision,
                         void *M, int ld, void *stream);

/* Same result as pbg_dev_smith_matrix, for callers that cannot allocate device
 * memory (an application whose own memory manager holds all of it, or a step
 * loop that must not hit the device-wide synchronisation of cudaMalloc/cudaFree).
 * No counterpart in the reference: it is an addition of this library.
 * All scratch lives in one fixed array inside the library (about 4.3 MiB held
 * by every GPU that loads it, until exit); nothing is allocated.  Limits:
 * at most 4096 real-space images, 2048 reciprocal half-vectors and
 * n_beads * (reciprocal half-vectors) * 16 bytes <= 4 MiB of phase tables
 * (e.g. 4096 beads at ewald_imag = 4); larger inputs (checked before any
 * table is built) return PBG_ERR_ARG.  The lattice tables reach the array as
 * kernel launch parameters, so no host buffer is staged and the host does not
 * wait for the stream.  The first call on a device looks up the array's device
 * address (make it before any stream capture).  Every call reuses the same
 * array, so calls that overlap on the GPU (different streams, or several host
 * threads) race; each call rewrites the parts it reads before reading them. */
PBG_API int pbg_dev_smith_matrix_noalloc(const double *pos, const double *radii, int n_beads,
                                         double box_length, double alpha, int m_max, int n_max,
                                         double scale, int precision, void *M, int ld, void *stream);

/* JO lubrication correction (diff_tensor.c:346-479) from positions, scaled
 * by `scale` and ADDED into M (M += scale * C). */
PBG_API int pbg_dev_lubrication_add(const double *pos, const double *radii, int n_beads,
                            double box_length, double cutoff, int cichocki, double scale,
                            double *M, int ld, void *stream);

/* Overlap flag (bead.c:169-260) from device positions; conn may be NULL
 * (no bonds).  The flag is written to *flag_dev (int, device). */
PBG_API int pbg_dev_check_overlaps(const double *pos, const double *radii, int n_beads,
                           double box_length, double threshold, const int *conn,
                           int *flag_dev, void *stream);

/* In-place lower Cholesky factor of an SPD matrix of order n (row-major,
 * leading dimension ld >= round_up(n, 64), rows/cols n..ld-1 are used as
 * padding).  precision selects FP64, the mixed FP32 path (float*; FP32
 * diagonal tiles, 3xTF32 trailing updates on the tcgen05 tensor cores) or
 * PBG_PREC_MIXED_FP64_DIAG.  Replaces np.linalg.cholesky (box.py:554).
 * info_dev (int, device) receives 0 or 1 + the index of the first
 * non-positive pivot. */
PBG_API int pbg_dev_cholesky(void *A, int n, int ld, int precision, int *info_dev, void *stream);

/* In-place inverse of an SPD FP64 matrix via its Cholesky factor: one
 * data-flow launch factors A and forms X = inv(L), then X^T X.  Replaces
 * np.linalg.inv (box.py:514,524,537). */
PBG_API int pbg_dev_spd_inverse(double *A, int n, int ld, int *info_dev, void *stream);

/* ---- system handle -------------------------------------------------- */
#define PBG_HI_NONE 0
#define PBG_HI_RPY 1
#define PBG_HI_RPY_SMITH 2
#define PBG_HI_RPY_LUB 3
#define PBG_HI_RPY_SMITH_LUB 4

#define PBG_PREC_FP64 0
#define PBG_PREC_MIXED 1
/* pbg_dev_cholesky only: an FP32 matrix (as PBG_PREC_MIXED) whose 64 x 64
 * diagonal tiles are factored and inverted in FP64 instead of FP32 (the
 * factorisation the lubricated mixed path uses for its resistance matrices). */
#define PBG_PREC_MIXED_FP64_DIAG 2

#define PBG_SCHEME_ERMAK 0
#define PBG_SCHEME_MIDPOINT 1

/* Matrix selectors for pbg_get_matrix. */
#define PBG_MAT_D 0
#define PBG_MAT_B 1
#define PBG_MAT_MFF 2
#define PBG_MAT_RFF 3
#define PBG_MAT_R 4

typedef struct pbg_params {
  int n_beads;
  int hydrodynamics;       /* PBG_HI_* */
  int precision;           /* PBG_PREC_* */
  int propagation_scheme;  /* PBG_SCHEME_* */
  double box_length;       /* Angstrom */
  double kBT;              /* J (Boltzmann * T) */
  double viscosity;        /* P */
  double ewald_alpha;
  int ewald_real;
  int ewald_imag;
  double lubrication_cutoff;
  int cichocki_correction;
  int check_overlaps;
  double overlap_treshold;
  int max_move_attempts;
  double m_midpoint;
} pbg_params;

typedef struct pbg_system pbg_system;

typedef struct pbg_step_report {
  long long draws_consumed;   /* normals consumed from the pool */
  long long steps_done;       /* steps fully completed */
  int last_attempts;          /* attempts taken by the last completed step */
  int max_attempts;           /* most attempts any step took */
  unsigned device_errors;     /* raw device error bits */
  int status;                 /* PBG_OK or PBG_ERR_* */
} pbg_step_report;

PBG_API int pbg_create(const pbg_params *params, pbg_system **out);
PBG_API int pbg_destroy(pbg_system *sys);

/* Copy state in (device pointers): positions N*3, radii N, connection
 * matrix N*N int32 (NULL: no bonds), force 3N (NULL: zero). */
PBG_API int pbg_set_state(pbg_system *sys, const double *pos, const double *radii, const int *conn,
                  void *stream);
PBG_API int pbg_set_force(pbg_system *sys, const double *force, void *stream);
/* Replaces the positions only (N*3, host or device), keeping radii and bonds. */
PBG_API int pbg_set_positions(pbg_system *sys, const double *pos, void *stream);
/* Divergence term of the lubricated diffusion matrix (box.py:211-215,
 * 560-610; JSON "divergence_term"): in the rpy_lub / rpy_smith_lub modes with
 * the Ermak scheme, pbg_step_begin adds div(D) dt after the deterministic
 * step, div(D) by forward differences (eps = 1e-7, 3N rebuilds of D). */
PBG_API int pbg_set_divergence(pbg_system *sys, int on);

/* Immobile beads (box.py:649-668; JSON "immobile_labels").  The system's
 * n_beads are the mobile beads; D, B and the noise cover them only, as in the
 * reference.  Immobile beads enter the overlap test (bead.c:169-218 over all
 * beads) and the inter-bead forces.  Host or device pointers:
 *   pos, radii   n_immobile x 3 and n_immobile doubles;
 *   order        n_beads + n_immobile ints: each bead's index in the caller's
 *                full bead list, mobile beads first (NULL: mobile beads come
 *                first in that list); it fixes the sign convention of the
 *                overlap test's pair vectors, as bead.c:180-182 does;
 *   conn_mi      n_beads x n_immobile int32 bond flags (NULL: none).
 * Call again to replace; n_immobile = 0 removes them. */
PBG_API int pbg_set_immobile(pbg_system *sys, int n_immobile, const double *pos, const double *radii,
                             const int *order, const int *conn_mi, void *stream);

/* Inter-bead forces on the device (interactions.py:483-821): Lennard-Jones
 * between all bead pairs, harmonic bonds and harmonic angles.  Bead indices
 * are combined: 0..n_beads-1 the mobile beads, n_beads.. the immobile ones.
 * Each bond and angle term appears once, in the order the reference's loops
 * meet it (interactions.py:185-247, 291-414), with the pair-vector form those
 * loops use.  The force of a step is the pbg_set_force vector plus
 * unit_scale times these terms, evaluated at the step-start positions by
 * pbg_step_begin; the energy (interaction units, like the reference's Box.E)
 * is read with pbg_get_energy.  Arrays may be host or device memory. */
#define PBG_LJ_NONE 0
#define PBG_LJ_6 6      /* LJ_6_attractive (interactions.py:711-745) */
#define PBG_LJ_12 12    /* LJ_12_repulsive (interactions.py:747-781) */
#define PBG_LJ_6_12 612 /* LJ_6_12 (interactions.py:783-821) */
/* Pair-vector forms of an angle term (interactions.py:291-414); P(a,b) is
 * the minimum-image vector from bead a to bead b. */
#define PBG_ANGLE_DIRECT 0    /* p12 = P(i,j), p23 = P(j,k) */
#define PBG_ANGLE_P23_DIFF 1  /* p23 = P(i,k) - P(i,j)  (j, k immobile) */
#define PBG_ANGLE_P12_DIFF 2  /* p12 = P(i,k) - P(j,k)  (i, j immobile) */
typedef struct pbg_interactions {
  int lennard_jones;               /* PBG_LJ_* */
  double lennard_jones_alpha;
  const double *hard_core_radius;  /* n_beads + n_immobile */
  const double *epsilon_lj;        /* n_beads + n_immobile */
  int n_bonds;
  const int *bonds;                /* 2 per bond: a, b; F_a += f, F_b -= f (mobile ends) */
  const double *bond_params;       /* 2 per bond: dist_eq [A], force_constant */
  int n_angles;
  const int *angles;               /* 4 per angle: i, j, k, PBG_ANGLE_* form */
  const double *angle_params;      /* 2 per angle: angle_eq [deg], force_constant */
  double unit_scale;               /* 1 (joule), 6.9477e-21 (kcal/mol), 1.602176634e-19 (eV) */
} pbg_interactions;
/* NULL removes the interactions. */
PBG_API int pbg_set_interactions(pbg_system *sys, const pbg_interactions *desc);
/* Interaction energy at the start of the last step (0 without interactions). */
PBG_API int pbg_get_energy(pbg_system *sys, double *energy_host, void *stream);
/* Force vector (3N, joules) used by the last step. */
PBG_API int pbg_get_force(pbg_system *sys, double *force_host, void *stream);
PBG_API int pbg_get_positions(pbg_system *sys, double *pos_out, void *stream);
/* Copy matrix `which` (PBG_MAT_*) as a dense row-major 3N x 3N FP64 array
 * (host or device memory; host output synchronises the stream). */
PBG_API int pbg_get_matrix(pbg_system *sys, int which, double *out, void *stream);

/* Overwrite matrix `which` from a dense row-major 3N x 3N FP64 array in host
 * or device memory (restart
 * files carry D, B, Mff, Rff and R; the mixed path rounds to FP32). */
PBG_API int pbg_set_matrix(pbg_system *sys, int which, const double *src, void *stream);

/* One Box.propagate (box.py:150-198) with host-driven attempts: the caller
 * supplies one noise vector per attempt through the callback-free protocol
 * pbg_step_begin / pbg_step_attempt / pbg_step_end. */
PBG_API int pbg_step_begin(pbg_system *sys, double dt, int build_Dff, int build_Dnf, int cholesky,
                   void *stream);
/* Runs one attempt with noise xi (device, 3N).  *accepted_host receives 1 if
 * the move was accepted (the call synchronises the stream). */
PBG_API int pbg_step_attempt(pbg_system *sys, const double *xi, int *accepted_host, void *stream);
PBG_API int pbg_step_end(pbg_system *sys, void *stream);
/* pbg_step_end, and the wrapped positions (N*3 doubles) copied to host memory
 * pos_host within the same synchronisation (one wait instead of two). */
PBG_API int pbg_step_finish(pbg_system *sys, double *pos_host, void *stream);

/* Multi-step run: steps j0 .. j0+n_steps-1 with the build cadence of
 * BD.py:177 (j % diff_freq == 0 ...), each step as Box.propagate does it.
 * Noise is consumed in order from `pool` (device or host, pool_len doubles);
 * each attempt takes 3N, so a pool filled from RandomState(seed) reproduces
 * the reference's trajectory.  With a host pool (or the midpoint scheme,
 * lubrication or the divergence term) the accept decision of each attempt
 * synchronises the stream, as pbg_step_attempt does.  With a device pool and
 * the Ermak scheme the attempts run on the device: from the second step with
 * the same flags, dt and force state a step is one CUDA graph launch (its
 * attempts under a conditional WHILE node) and one wait; the results are the
 * same bit for bit.  Changing the system (pbg_set_state, pbg_set_immobile,
 * pbg_set_interactions, pbg_set_divergence) drops that graph.  A step that runs out of
 * noise (PBG_ERR_NOISE) or of move attempts (PBG_ERR_ATTEMPTS, box.py:248)
 * is rolled back to its start positions and ends the run; pbg_run_report
 * gives the steps completed, the noise consumed and the attempt counts. */
PBG_API int pbg_run(pbg_system *sys, long long j0, int n_steps, double dt, int diff_freq, int lub_freq,
            int chol_freq, const double *pool, long long pool_len, void *stream);
PBG_API int pbg_run_report(pbg_system *sys, pbg_step_report *out, void *stream);

/* ---- Tier 3: batched replicas -------------------------------------------
 * No counterpart in the reference, which advances one Box per process.  A
 * batch holds many independent BD systems (rpy or rpy_smith hydrodynamics,
 * Ermak scheme, one precision and Ewald parameter set for all) and advances
 * them together; each replica follows Box.propagate (box.py:150-250) on its
 * own positions, radii, box, temperature and noise.  Replicas can be added
 * and removed between steps; slot ids stay valid until removal.  Arrays
 * indexed by slot (mask, accepted, status) have pbg_batch_slots() entries.
 * A step: pbg_batch_step_begin, then for the replicas still moving noise
 * (pbg_batch_set_noise or pbg_batch_fill_noise) and pbg_batch_step_attempt
 * until each is accepted (box.py:219-248), then pbg_batch_step_end. */
typedef struct pbg_batch pbg_batch;

/* precision, hydrodynamics, propagation_scheme and the Ewald fields of tmpl
 * apply to every replica. */
PBG_API int pbg_batch_create(const pbg_params *tmpl, pbg_batch **out);
PBG_API int pbg_batch_destroy(pbg_batch *b);
/* Device bytes one replica of n_beads takes (matrices, factor, tables, state). */
PBG_API long long pbg_batch_footprint(int precision, int hydrodynamics, int ewald_imag, int n_beads);
/* p: n_beads, box_length, kBT, viscosity, check_overlaps, overlap_treshold,
 * max_move_attempts (pbg_batch_step; at least 1).
 * pos (3N), radii (N): host or device memory. */
PBG_API int pbg_batch_add(pbg_batch *b, const pbg_params *p, const double *pos, const double *radii, int *slot);
PBG_API int pbg_batch_remove(pbg_batch *b, int slot);
PBG_API int pbg_batch_slots(pbg_batch *b);
PBG_API int pbg_batch_set_positions(pbg_batch *b, int slot, const double *pos);
PBG_API int pbg_batch_get_positions(pbg_batch *b, int slot, double *out);
/* The same copy ordered on `stream` without waiting for it (out: pinned host
 * memory for the copy to be asynchronous). */
PBG_API int pbg_batch_get_positions_async(pbg_batch *b, int slot, double *out, void *stream);
/* External force (3N), or NULL for none. */
PBG_API int pbg_batch_set_force(pbg_batch *b, int slot, const double *F);
/* Noise of the next attempt (3N normals, host or device memory). */
PBG_API int pbg_batch_set_noise(pbg_batch *b, int slot, const double *xi);
/* Counter-based device noise (Philox-4x32-10 + Box-Muller): stream position
 * `draws` of the stream `seed`; pbg_batch_fill_noise fills the masked
 * replicas and advances each stream by 3N draws (rounded up to even). */
PBG_API int pbg_batch_set_seed(pbg_batch *b, int slot, unsigned long long seed, unsigned long long draws);
PBG_API int pbg_batch_get_draws(pbg_batch *b, int slot, unsigned long long *draws);
PBG_API int pbg_batch_fill_noise(pbg_batch *b, const unsigned char *mask, void *stream);
PBG_API int pbg_batch_step_begin(pbg_batch *b, double dt, int build_D, int cholesky, void *stream);
PBG_API int pbg_batch_step_attempt(pbg_batch *b, const unsigned char *mask, unsigned char *accepted, void *stream);
/* status[slot]: 0, the first non-positive pivot (1-based), or -1 (a wait gave up). */
PBG_API int pbg_batch_step_end(pbg_batch *b, int *status, void *stream);
/* One whole step of every replica, all of whose noise comes from the
 * counter-based device streams (pbg_batch_set_seed): the start of the step
 * (as pbg_batch_step_begin), then rounds of attempts -- each replica still
 * moving draws 3N normals, moves by sqrt(2 dt) B xi, is tested for overlaps
 * and, on an overlap, moved back -- until every replica is accepted or has
 * used max_move_attempts (pbg_params of pbg_batch_add), then the wrap into
 * the box.  The rounds run on the device under a conditional WHILE node of
 * the step's CUDA graph (captured once a step repeats with the same
 * membership, flags and dt; a launch runs at most 4096 rounds, further
 * rounds are launched from the host), so a repeated step is one graph launch
 * and one synchronisation.  Each replica's noise, moves and decisions are
 * those of the attempt-by-attempt path with pbg_batch_fill_noise.
 * status[slot] as pbg_batch_step_end; attempts[slot] (may be NULL) receives
 * the attempts each replica took.  PBG_ERR_ATTEMPTS when a replica ran out of
 * attempts (its last move undone; box.py:248 asserts), then PBG_ERR_BARRIER /
 * PBG_ERR_NOT_SPD as pbg_batch_step_end.  No counterpart in the reference.
 * A batch's calls are ordered on the stream they are given: use one stream
 * per batch. */
PBG_API int pbg_batch_step(pbg_batch *b, double dt, int build_D, int cholesky, int *status, int *attempts,
                           void *stream);
/* D or B (PBG_MAT_D / PBG_MAT_B) of one replica, 3N x 3N FP64 row-major host array. */
PBG_API int pbg_batch_get_matrix(pbg_batch *b, int slot, int which, double *out);
/* Factors a copy of one replica's current D with the single-matrix
 * factorisation (the batch's precision); *info as status[] of
 * pbg_batch_step_end.  After a step that reported a failed factorisation it
 * tells a matrix that is not positive definite (info > 0 again) from one the
 * batched factorisation failed on (info 0).  The batch is left unchanged. */
PBG_API int pbg_batch_check_factor(pbg_batch *b, int slot, int *info, void *stream);

/* Schedule of the batched factorisation (no counterpart in the reference).
 * merge_order: how the replicas' task segments are interleaved in the one
 * task list; ctas_per_sm: resident CTAs per SM of the persistent kernel
 * (0 = as many as fit; a larger count is cut to what fits).  No choice
 * changes any result bit.  The mixed batch factors left-looking (tasks per
 * column: the diagonal pair and the updates, then the solves), the FP64 batch
 * right-looking (tasks per panel: F, updates, solves); the segments merged are
 * those. */
enum {
  PBG_MERGE_LARGER_FIRST = 0,
  PBG_MERGE_ADDED = 1,
  PBG_MERGE_SMALLER_FIRST = 2,
  PBG_MERGE_REPLICA_MAJOR = 3,
  /* larger first, in consecutive chunks of replicas whose matrices together
   * fit 32 / 64 / 128 MiB (the chunks' segments interleaved within a chunk,
   * chunk after chunk), so that a tile is still in L2 for its next update */
  PBG_MERGE_CHUNK_32M = 4,
  PBG_MERGE_CHUNK_64M = 5,
  PBG_MERGE_CHUNK_128M = 6
};
#define PBG_MERGE_ORDERS 7
PBG_API int pbg_batch_set_schedule(pbg_batch *b, int merge_order, int ctas_per_sm);
/* Autotuner: after a step has built D (not inside a step), times `reps`
 * factorisations of the current matrices under every schedule (the
 * PBG_MERGE_ORDERS merge orders x 1 .. min(2, the kernel's residency) CTAs
 * per SM),
 * keeps the fastest and leaves B as the factor of the current D (the value a
 * step would give).  best[2] = {merge_order, ctas_per_sm}; ms (may be NULL)
 * receives the mean time of each candidate, merge order major
 * (2 * PBG_MERGE_ORDERS entries; -1 for a candidate not run). */
PBG_API int pbg_batch_autotune(pbg_batch *b, int reps, int *best, float *ms, void *stream);
/* One replica's factorisation task list (host only, no device needed; no
 * counterpart in the reference): for an nt x nt tile grid in the batch's
 * precision, tasks[4 t .. 4 t + 3] = (kind, i, j, k) of task t (cap tasks at
 * most) and seg[s] the start of segment s (the last entry is the end; seg_cap
 * entries at most).  The mixed list is left-looking (kinds 0 diagonal pair,
 * 1 update pair, 2 solve pair; rows i and i + 1 of column j), the FP64 list
 * right-looking (kinds 0 F, 1 S, 2 U, 4 U of rows i and i + 1; panel k).
 * *n_tasks and *n_segs receive the counts; PBG_ERR_ARG if either does not
 * fit or nt < 1. */
PBG_API int pbg_cholesky_task_list(int nt, int precision, int *tasks, int cap, int *seg, int seg_cap,
                                   int *n_tasks, int *n_segs);
/* How the start of a step (Ewald build, copy into B, factorisation,
 * deterministic move) -- or with pbg_batch_step the whole step -- runs:
 * 1 = one CUDA graph launch (captured once a step
 * repeats with the same membership, flags and dt), 0 = its kernels launched
 * one by one, -1 = the driver refused the capture (kernels launched one by
 * one from then on).  No counterpart in the reference. */
PBG_API int pbg_batch_graph_state(pbg_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* PYBROWN_B200_H */
