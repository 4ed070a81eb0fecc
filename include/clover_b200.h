/*
 * Native API of the B200 hydro-cycle engine: a whole CloverLeaf3D chunk kept
 * resident in HBM and advanced by the device, with dt, time and the step
 * count on the GPU and the step replayed from CUDA graphs.
 *
 * This is the fast path behind the drop-in ABI of clover_kernels.h: the same
 * kernels, sequenced as hydro.f90:46-192 sequences the *_kernel calls, but
 * with no host round trip per step. The deck reader mirrors parse.f90 and
 * read_input.f90 (same keywords, same defaults).
 */
#ifndef CLOVER_B200_H
#define CLOVER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLOVER_MAX_STATES 16

/* The keys of a *clover deck (read_input.f90:38-86 defaults). State bounds
 * are stored as written in the deck; the nudge by a hundredth of a cell
 * (read_input.f90:287-303) is applied when a chunk is created. */
typedef struct clover_deck {
  int x_cells, y_cells, z_cells;
  double xmin, ymin, zmin, xmax, ymax, zmax;
  double initial_timestep, max_timestep, timestep_rise, end_time;
  double dtmin, dtc_safe, dtu_safe, dtv_safe, dtw_safe, dtdiv_safe;
  int end_step, summary_frequency, visit_frequency, tiles_per_chunk;
  int test_problem, profiler_on;
  int number_of_states;
  int state_defined[CLOVER_MAX_STATES];
  double state_density[CLOVER_MAX_STATES], state_energy[CLOVER_MAX_STATES];
  double state_xvel[CLOVER_MAX_STATES], state_yvel[CLOVER_MAX_STATES];
  double state_zvel[CLOVER_MAX_STATES];
  double state_xmin[CLOVER_MAX_STATES], state_xmax[CLOVER_MAX_STATES];
  double state_ymin[CLOVER_MAX_STATES], state_ymax[CLOVER_MAX_STATES];
  double state_zmin[CLOVER_MAX_STATES], state_zmax[CLOVER_MAX_STATES];
  double state_radius[CLOVER_MAX_STATES];
  int state_geometry[CLOVER_MAX_STATES]; /* 1 cuboid, 2 sphere, 3 point */
} clover_deck;

/* read_input.f90:38-86 defaults (no states). */
void clover_deck_defaults(clover_deck *deck);
/* Parse the text of a deck (the *clover ... *endclover block). Returns 0, or
 * a nonzero code with a message in err: 1 no states, 2 state defined twice,
 * 3 bad number, 4 too many states. */
int clover_deck_parse(const char *text, clover_deck *deck, char *err, int errlen);

typedef struct clover_chunk clover_chunk;

#define CLOVER_PRECISION_FP64 0  /* every field FP64: the parity path */
#define CLOVER_PRECISION_MIXED 1 /* FP32 storage, FP64 density/mass flux/work */

/* Build the chunk on the current device: allocate, initialise_chunk,
 * generate_chunk, ideal_gas, the depth-2 halo prime and the step-0 field
 * summary (start.f90:49-136). NULL on failure (see clover_last_error). */
clover_chunk *clover_chunk_create(const clover_deck *deck, int precision);
void clover_chunk_destroy(clover_chunk *c);
const char *clover_last_error(void);

/* Enqueue n hydro steps (hydro.f90:46-84 minus the end test) on the chunk
 * stream, with field summaries at the deck's summary_frequency. Returns
 * immediately. Uses CUDA graphs when enabled (the default). */
int clover_chunk_step(clover_chunk *c, int n);
/* The hydro loop of hydro.f90 to completion (end_step or end_time), with
 * the final field summary. Returns the number of steps taken, or <0 on the
 * small-timestep error. */
int clover_chunk_run(clover_chunk *c);
/* Wait for the chunk stream. */
int clover_chunk_sync(clover_chunk *c);
/* 0 = launch kernels directly, 1 = replay captured graphs. */
void clover_chunk_use_graphs(clover_chunk *c, int on);
/* 1 (default) = the fused kernels, 0 = one kernel per reference loop nest.
 * Both give the same results bit for bit. Only before the first step. */
void clover_chunk_use_fused(clover_chunk *c, int on);
/* 1 (default) = the fused step's stencils that stage their input planes in
 * shared memory with bulk-tensor (TMA) copies, where the chunk could make
 * their tensor maps; 0 = their register-marching forms. Both give the same
 * results bit for bit. Returns 1 if the staged forms are in use. Ensembles
 * always use the register-marching forms. */
int clover_chunk_use_tma(clover_chunk *c, int on);

/* Self-test of the staged kernels' failure detection (no counterpart in the
 * reference): a one-block kernel waits, with the bounded wait those kernels
 * use and a limit of `cycles` SM clocks, for copies that nothing issues, and
 * reports as they do. Returns CLOVER_STATUS_TIMEOUT when the wait ran out
 * and was reported (the expected answer), 0 if it did not run out, or
 * CLOVER_STATUS_CUDA_ERROR. The device stays usable. */
int clover_gpu_wait_selftest(long long cycles);

/* Self-test of the correctly rounded FP64 quotient the step kernels form from
 * one approximate reciprocal per divisor (no counterpart in the reference,
 * whose divisions are IEEE divisions): q[i] = x[i] / b[i] for n host values,
 * through that quotient where x[i] and b[i] lie in its range (fast[i] = 1)
 * and by IEEE division elsewhere (fast[i] = 0). Either way q[i] must equal
 * the IEEE quotient bit for bit. Returns 0 or CLOVER_STATUS_CUDA_ERROR. */
int clover_gpu_quotient_selftest(const double *x, const double *b, double *q, int *fast,
                                 long long n);

/* Host copies of the device records (these synchronise):
 * steps taken, simulated time, dt of each step, field summaries
 * (vol, mass, ie, ke, press) with the step each was taken at. */
int clover_chunk_steps(clover_chunk *c);
double clover_chunk_time(clover_chunk *c);
int clover_chunk_dt_history(clover_chunk *c, double *out, int cap);
int clover_chunk_summaries(clover_chunk *c, double *out5, int *steps, int cap);
/* Device status bits (CLOVER_STATUS_* of clover_kernels.h). */
int clover_chunk_status(clover_chunk *c);

/* Copy one field (reference field id 1..19, data.f90:55-74) into a host
 * array in the reference layout, widening FP32 storage to FP64. */
int clover_chunk_read_field(clover_chunk *c, int field_id, double *host);
/* Replace one field from a host array in the reference layout. */
int clover_chunk_write_field(clover_chunk *c, int field_id, const double *host);

/* The chunk stream (a cudaStream_t), for timing with events on it. */
uintptr_t clover_chunk_stream(clover_chunk *c);
/* Device bytes held by the chunk. */
long long clover_chunk_device_bytes(clover_chunk *c);
/* Profile mode: when on, steps launch kernels directly and every kernel
 * group is bracketed by events on the chunk stream. The report returns, per
 * group (names[i*name_len], NUL-terminated): summed ms, summed algorithmic
 * bytes (distinct 3D arrays read + written x cells x element size) and
 * launches since the last report, then resets. Turning it off clears it. */
void clover_chunk_profile(clover_chunk *c, int on);
int clover_chunk_profile_report(clover_chunk *c, char *names, int name_len, double *ms,
                                double *bytes, int *launches, int cap);
/* Kernel launches one hydro step issues (graph nodes per step). */
int clover_chunk_launches_per_step(clover_chunk *c);

/* VTK output as visit.f90 writes it (legacy ASCII rectilinear grids of
 * density, energy, pressure, viscosity and the node velocities, Fortran
 * E12.4, plus the clover.visit index) into dir (default "."). With a deck's
 * visit_frequency set, a run writes at step 0 (when the first step is
 * enqueued), every visit_frequency steps and at the end, a writer thread formatting each frame while the GPU steps
 * on; clover_chunk_visit writes the current step and waits for the file.
 * Ensembles write one file per deck (chunk number = deck + 1). */
int clover_chunk_set_visit_dir(clover_chunk *c, const char *dir);
int clover_chunk_visit(clover_chunk *c);
/* E12.4 formatting of one value into out (13 bytes), for tests. */
int clover_format_e12_4(double v, char *out13);

/* Checkpoint / restart of a chunk or ensemble (no counterpart in the
 * reference, which restarts from the deck only). The file holds every device
 * array of the chunk byte for byte plus the step state (dt, time, step, the dt
 * and summary histories); restoring it into a chunk made from the same decks
 * and precision continues bit for bit as if the run had not stopped. 0 on
 * success; negative on I/O errors or a checkpoint that does not match. */
int clover_chunk_checkpoint(clover_chunk *c, const char *path);
int clover_chunk_restore(clover_chunk *c, const char *path);

/* ---- Ensembles: many independent decks advanced together ----
 * No counterpart in the reference (which runs one deck per job). The decks
 * of an ensemble may differ in size, states and timestep controls; each
 * keeps its own dt, time and calc_dt reduction, and nothing synchronises
 * one deck with another. Their arrays share one device allocation per
 * field, and every kernel of the (fused) step runs once over all decks: a
 * persistent grid of blocks walks a schedule of (deck, tile) items. The
 * decks must share end_step, summary_frequency and calc_dt's safety factors
 * (one step sequence); end_time is not applied per deck.
 * clover_chunk_step/run/sync/stream/profile/use_graphs work on ensembles
 * (run advances every deck end_step steps); the per-deck results come from
 * the clover_ensemble_* calls. */
clover_chunk *clover_ensemble_create(const clover_deck *decks, int n_decks, int precision);
int clover_ensemble_decks(clover_chunk *c);
/* Time candidate schedules (item order, grid size, marching segment length)
 * per batched launch over trial_steps steps each, keep the fastest, then
 * reset the ensemble to its initial state. Returns the number of launches
 * tuned, -1 on error. */
int clover_ensemble_autotune(clover_chunk *c, int trial_steps);
/* Set every deck up again (step 0); the tuned schedules stay. */
int clover_ensemble_reset(clover_chunk *c);
/* One schedule for every batched launch instead of the tuned ones: item
 * order (0 deck order, 1 largest deck first, 2 round robin), grid_div (0 one
 * block per item, n: resident blocks / n), seg (marching segment length, 0
 * the default). */
int clover_ensemble_set_schedule(clover_chunk *c, int order, int grid_div, int seg);
/* The schedule in use, one line per launch: key order grid_div seg blocks
 * items. Returns the length of the full text. */
int clover_ensemble_schedule(clover_chunk *c, char *buf, int len);
int clover_ensemble_status(clover_chunk *c, int deck);
double clover_ensemble_time(clover_chunk *c, int deck);
int clover_ensemble_dt_history(clover_chunk *c, int deck, double *out, int cap);
int clover_ensemble_summaries(clover_chunk *c, int deck, double *out5, int *steps, int cap);
int clover_ensemble_read_field(clover_chunk *c, int deck, int field_id, double *host);

/* ---- Host driver over the drop-in ABI ----
 * The reference's own control flow (start.f90, hydro.f90, timestep.f90,
 * PdV.f90, advection.f90) over host arrays allocated as build_field.f90
 * allocates them, every kernel call going through clover_kernels.h. Its
 * destroy call releases every mirror of the process. */
typedef struct clover_dropin clover_dropin;
clover_dropin *clover_dropin_create(const clover_deck *deck);
/* Run the hydro loop to its end (deck end_step/end_time, or max_steps).
 * Returns the steps taken, negative on the small-timestep error. */
int clover_dropin_run(clover_dropin *d, int max_steps);
int clover_dropin_dt_history(clover_dropin *d, double *out, int cap);
int clover_dropin_summaries(clover_dropin *d, double *out5, int *steps, int cap);
/* Copy a field (id 1..19) back to the host and out (n elements, reference layout). */
int clover_dropin_read_field(clover_dropin *d, int field_id, double *out, long long n);
void clover_dropin_destroy(clover_dropin *d);

/* ---- Brick decomposition of one deck (clover.f90's MPI layer) ----
 * clover_decompose, clover.f90:108-256: the chunk grid chunks_xyz[3] for
 * n_chunks chunks, and per chunk (ids 1..n in x-fastest order) its global
 * cell range extents[6*i..] = left, right, bottom, top, back, front and its
 * neighbours[6*i..] (left, right, bottom, top, back, front; -1 = external
 * face). Host only. Returns 0, or -1 when a chunk would be empty. */
int clover_decompose(int x_cells, int y_cells, int z_cells, int n_chunks, int *chunks_xyz,
                     int *extents, int *neighbours);
/* The decomposed run of the reference over n_chunks bricks of one deck in
 * this process: the drop-in driver's control flow on every brick, each
 * update_halo exchanging the bricks' faces on the device (pack_kernel.f90's
 * messages, x then y then z) before the reflective halos of the external
 * faces, dt the minimum over the bricks (clover_min), the summaries their sum
 * (clover_sum). NULL on failure (clover_gpu_error_string). */
typedef struct clover_bricks clover_bricks;
clover_bricks *clover_bricks_create(const clover_deck *deck, int n_chunks);
/* The transport of a decomposed run with one brick per rank (the reference's
 * MPI model): implemented by the caller, e.g. over torch.distributed.
 * exchange: one axis phase of clover_exchange (axis 0 x, 1 y, 2 z): send
 * send_lo (n_lo doubles) to chunk lo and receive recv_lo from it, the same
 * with chunk hi; a chunk of -1 is no neighbour (nothing to move). Chunk ids
 * are ranks + 1. min: clover_min of one value in place; sum: clover_sum of n
 * values in place. Each returns 0 on success. host_staged: 1 = the message
 * buffers are host (pinned) memory, 0 = device memory, filled and drained on
 * the library's stream, which is idle during the call. */
typedef struct clover_transport {
  void *ctx;
  int host_staged;
  int (*exchange)(void *ctx, int axis, int lo, double *send_lo, double *recv_lo, long long n_lo,
                  int hi, double *send_hi, double *recv_hi, long long n_hi);
  int (*min)(void *ctx, double *v);
  int (*sum)(void *ctx, double *v, int n);
} clover_transport;
/* This rank's brick (chunk rank + 1 of clover_decompose's n_chunks) of the
 * decomposed run; every rank calls it with the same deck and n_chunks. The
 * brick queries below then address the one local brick as brick 0. */
clover_bricks *clover_bricks_create_rank(const clover_deck *deck, int n_chunks, int rank,
                                         const clover_transport *t);
int clover_bricks_run(clover_bricks *w, int max_steps);
/* Number of bricks; chunks_xyz gets the chunk grid. */
int clover_bricks_count(clover_bricks *w, int *chunks_xyz);
/* Global cell range and neighbours of brick (0-based). */
int clover_bricks_extent(clover_bricks *w, int brick, int *ext6, int *neighbours6);
int clover_bricks_dt_history(clover_bricks *w, double *out, int cap);
int clover_bricks_summaries(clover_bricks *w, double *out5, int *steps, int cap);
/* Field id 1..19 of a brick in its reference layout (n elements). */
int clover_bricks_read_field(clover_bricks *w, int brick, int field_id, double *out, long long n);
void clover_bricks_destroy(clover_bricks *w);

#ifdef __cplusplus
}
#endif
#endif
