/*
 * sb2.h — C ABI of the B200-native Synergia space-charge + tracking step.
 *
 * Every entry point takes plain pointers and sizes.  Particle storage follows
 * the reference Bunch contract: an N x 7 FP64 column-major array (columns x,
 * xp, y, yp, cdt, dpop, id; column stride = capacity) plus a uint8 mask per
 * particle (1 = alive); lost particles are never compacted.
 *
 * Reference interfaces replaced (paths inside the synergia2 project):
 *   Space_charge_3d_open_hockney_options  simulation/implemented_collective_options.h:67-126
 *   Space_charge_3d_open_hockney::apply_impl / apply_bunch
 *                                         collective/space_charge_3d_open_hockney.cc:400-453
 *   FF_element::apply(slice, bunch)       libFF/ff_element.h:25-67
 *   LibFF_operation::apply_impl           simulation/independent_operation.h:45-60
 *   Aperture_operation<AP>::apply_impl    simulation/aperture_operation.h:14-24
 *   Bunch::apply_aperture                 bunch/bunch.h:727-740
 *   Split_operator_stepper::apply_impl    simulation/split_operator_stepper.cc:132-261
 *   Split_operator_stepper_elements       simulation/split_operator_stepper_elements.cc:4-47
 *   Independent_stepper_elements          simulation/independent_stepper_elements.cc:3-36
 *   Propagator::propagate                 simulation/propagator.cc:157-283
 *   Core_diagnostics::calculate_mom2      bunch/core_diagnostics.cc:351-365
 *   calculate_emittances                  bunch/diagnostics_full2_host.cc
 *
 * Errors: every call returns an sb2_status; sb2_last_error() returns the
 * message of the last failure on the calling thread (the text the reference
 * throws as std::runtime_error where one exists).
 */
#ifndef SB2_H_
#define SB2_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t sb2_status;
enum {
    SB2_OK = 0,
    SB2_ERR_INVALID = 1,     /* bad argument / option */
    SB2_ERR_CUDA = 2,        /* CUDA runtime failure */
    SB2_ERR_RUNTIME = 3,     /* runtime_error raised by the physics (e.g. degenerate domain) */
    SB2_ERR_UNSUPPORTED = 4, /* valid in the reference, not supported by this build */
    SB2_ERR_NOMEM = 5        /* device allocation failed */
};

/* Message of the last failing call on this thread. */
const char* sb2_last_error(void);
/* Library version string. */
const char* sb2_version(void);
/* The library links the CUDA runtime statically: sb2_set_device selects the
 * GPU for this thread's later calls (as cudaSetDevice does for the caller's
 * own runtime; one process per GPU calls it with its local rank). */
sb2_status sb2_set_device(int32_t device);

/* Per-category device timing of the library's own launches, measured with
 * CUDA events recorded on the launching stream (the reference's
 * scoped_simple_timer regions, utils/simple_timer.h:50-66).  Categories:
 * 0 track (fused particle passes of drifts, thin kicks, apertures, the
 * space-charge kick), 1 domain (bookkeeping + domain), 2 deposit, 3 green
 * (Green-function transform), 4 solve (FFT convolution), 5 efield, 6 sort
 * (cell-ordered working copy), 7 track_full (particle passes with Yoshida
 * integrators or sector bends).  Off by default. */
sb2_status sb2_profile_enable(int32_t on);
sb2_status sb2_profile_read(int32_t category, const char** name, double* total_ms, int64_t* launches,
                            int32_t reset);

/* FP64 peak of the current device at its present clocks, in TFLOP/s (an FMA
 * counts 2): a kernel of independent FMA chains on every SM, best of six
 * timed launches on `stream` (CUDA events), synchronous.  The denominator of
 * the FP64-bound particle passes' roofline. */
sb2_status sb2_fp64_peak_probe(double* tflops, void* stream);

/* ---------------------------------------------------------------------
 * Options of the 3D open-boundary Hockney solver.
 * Replaces Space_charge_3d_open_hockney_options
 * (simulation/implemented_collective_options.h:67-126).
 * ------------------------------------------------------------------- */
enum { SB2_GREEN_POINTLIKE = 0, SB2_GREEN_LINEAR = 1 };
enum { SB2_PRECISION_FP64 = 0, SB2_PRECISION_MIXED = 1 };

typedef struct sb2_sc3d_options {
    int32_t shape[3];         /* grid (gx, gy, gz) */
    int32_t doubled_shape[3]; /* doubled grid; must be 2*shape */
    double size[3];           /* fixed-domain size [m, m, m(cdt)] */
    double offset[3];         /* fixed-domain offset */
    int32_t green_fn;         /* SB2_GREEN_* (default linear) */
    int32_t periodic_z;       /* not implemented in the reference (throws) */
    double z_period;
    int32_t grid_entire_period;
    double n_sigma;           /* adaptive domain size in sigmas (default 8) */
    double kick_scale;        /* default 1 */
    int32_t domain_fixed;     /* 1 after set_fixed_domain */
    int32_t comm_group_size;  /* accepted for API parity; single GPU */
    int32_t precision;        /* SB2_PRECISION_FP64 (drop-in) or _MIXED */
} sb2_sc3d_options;

/* Space_charge_3d_open_hockney_options(gridx, gridy, gridz) defaults. */
sb2_status sb2_sc3d_options_init(sb2_sc3d_options* opts, int gx, int gy, int gz);
/* Space_charge_3d_open_hockney_options::set_fixed_domain. */
sb2_status sb2_sc3d_options_set_fixed_domain(sb2_sc3d_options* opts, const double offset[3],
                                             const double size[3]);

/* ---------------------------------------------------------------------
 * Bunch: device-resident particles.  Replaces Bunch / bunch_particles_t
 * (bunch/bunch.h, bunch/bunch_particles.h:24-205).
 * ------------------------------------------------------------------- */
typedef struct sb2_bunch sb2_bunch;

/* Reference particle given as (charge [e], mass [GeV], value [GeV], kind):
 * kind 0 = total energy, 1 = momentum, 2 = kinetic energy. */
enum { SB2_REF_TOTAL_ENERGY = 0, SB2_REF_MOMENTUM = 1, SB2_REF_KINETIC_ENERGY = 2 };

/* Bunch(ref, total_num, real_num): allocates capacity = n particles on the
 * current device, ids 0..n-1, all masks 1, coordinates 0. */
sb2_status sb2_bunch_create(int32_t charge, double mass, double value, int32_t kind, int64_t n,
                            double real_num, sb2_bunch** out);
/* Borrow caller-owned device memory (no copy, no ownership): parts is N x 7
 * column-major with column stride `stride`, masks N bytes, discards N bytes
 * (may be NULL). */
sb2_status sb2_bunch_wrap(int32_t charge, double mass, double value, int32_t kind, double* parts,
                          int64_t stride, uint8_t* masks, uint8_t* discards, int64_t n,
                          double real_num, sb2_bunch** out);
sb2_status sb2_bunch_destroy(sb2_bunch* b);
/* checkin_particles: host N x 7 column-major (stride n) -> device; masks may
 * be NULL (all alive).  Recounts valid particles. */
sb2_status sb2_bunch_set_particles(sb2_bunch* b, const double* host_parts, const uint8_t* host_masks);
/* checkout_particles: device -> host; any output may be NULL. */
sb2_status sb2_bunch_get_particles(sb2_bunch* b, double* host_parts, uint8_t* host_masks,
                                   uint8_t* host_discards);
/* Device pointers of the bunch (for zero-copy callers). */
sb2_status sb2_bunch_device_arrays(sb2_bunch* b, double** parts, int64_t* stride, uint8_t** masks,
                                   uint8_t** discards);
/* n_active (size), n_valid (local_num), n_total, real_num. */
sb2_status sb2_bunch_counts(sb2_bunch* b, int64_t* n_active, int64_t* n_valid, int64_t* n_total,
                            double* real_num);
/* State [x, xp, y, yp, cdt, dpop] of the design reference particle and
 * s_n of the bunch reference particle. */
sb2_status sb2_bunch_design_state(sb2_bunch* b, double state[6], double* s_n);
/* Host-side state of a bunch beyond its particle arrays: the bunch and the
 * design reference particle (Reference_particle, foundation/
 * reference_particle.h: charge, four momentum, state, s, s_n, repetition),
 * the number of turns propagated and the particle counts kept by
 * update_total_num (bunch_particles.cc:388).  get + set restore a bunch
 * exactly, which is what a checkpoint needs (simulation/checkpoint.cc:18). */
typedef struct sb2_refpart_state {
    int32_t charge;
    int32_t repetition;
    double mass, gamma, beta, momentum, energy;
    double state[6];
    double s, s_n;
} sb2_refpart_state;
typedef struct sb2_bunch_state {
    sb2_refpart_state ref;    /* the bunch's reference particle */
    sb2_refpart_state design; /* the lattice (design) reference particle */
    int32_t design_set;       /* 0 until the first propagate call sets `design` */
    int32_t turns_done;
    int64_t n_valid, n_total;
    double real_num;
} sb2_bunch_state;
/* Current state (reads the device counters; synchronous). */
sb2_status sb2_bunch_get_state(sb2_bunch* b, sb2_bunch_state* out);
/* Restores a state taken by sb2_bunch_get_state (device counters included);
 * the mass and charge must match the bunch's. */
sb2_status sb2_bunch_set_state(sb2_bunch* b, const sb2_bunch_state* in);
/* Discard flags (bunch_particles.h:40), host N bytes -> device. */
sb2_status sb2_bunch_set_discards(sb2_bunch* b, const uint8_t* host_discards);
/* Stream-ordered copy of the resident particles, masks and discards (each
 * output may be NULL; give pinned host memory for a copy that does not
 * block) plus the device counts, enqueued on `stream` (cudaStream_t or NULL) behind the work
 * already queued there, without a host synchronisation.  A bunch that is
 * in its cell-ordered working copy is scattered back to the caller's order
 * on the device first and keeps using the working copy afterwards, so a
 * checkpoint costs one scatter and the copies; later propagate calls on
 * the same stream are ordered after it.  The counts of the snapshot are
 * read with sb2_bunch_snapshot_counts once the stream has reached it. */
sb2_status sb2_bunch_snapshot_async(sb2_bunch* b, double* host_parts, uint8_t* host_masks,
                                    uint8_t* host_discards, void* stream);
sb2_status sb2_bunch_snapshot_counts(sb2_bunch* b, int64_t* n_valid, int64_t* n_total, double* real_num);
/* Synthetic seeded 6D uncorrelated Gaussian on the device (zero means;
 * sigmas for x, xp, y, yp, cdt, dpop); counter-based generator, ids 0..n-1. */
sb2_status sb2_bunch_populate_gaussian(sb2_bunch* b, const double sigma[6], uint64_t seed);
/* Core_diagnostics::calculate_mean and calculate_mom2 (6 + 36 values,
 * divided by n_total) and the rms emittances sqrt(det 2x2) of the x, y, z
 * planes (diagnostics_full2_host.cc). */
sb2_status sb2_bunch_moments(sb2_bunch* b, double mean[6], double mom2[36], double emit[3]);

/* ---------------------------------------------------------------------
 * Lattice: element list with attributes.  Replaces Lattice /
 * Lattice_element (lattice/lattice.h, lattice/lattice_element.h) as the
 * input of the steppers; no MAD-X parsing.
 * ------------------------------------------------------------------- */
typedef struct sb2_lattice sb2_lattice;
sb2_status sb2_lattice_create(const char* name, sb2_lattice** out);
sb2_status sb2_lattice_destroy(sb2_lattice* l);
sb2_status sb2_lattice_set_reference_particle(sb2_lattice* l, int32_t charge, double mass,
                                              double value, int32_t kind);
/* Appends an element of MAD-X type name (drift, quadrupole, sbend,
 * multipole, sextupole, marker, monitor, ...); returns its index. */
sb2_status sb2_lattice_append(sb2_lattice* l, const char* type, const char* name, int32_t* index);
sb2_status sb2_lattice_set_double(sb2_lattice* l, int32_t index, const char* attr, double value);
sb2_status sb2_lattice_set_string(sb2_lattice* l, int32_t index, const char* attr, const char* value);
sb2_status sb2_lattice_set_vector(sb2_lattice* l, int32_t index, const char* attr, const double* v,
                                  int32_t n);
sb2_status sb2_lattice_length(sb2_lattice* l, double* length);
sb2_status sb2_lattice_num_elements(sb2_lattice* l, int32_t* n);

/* ---------------------------------------------------------------------
 * Propagator.  A stepper (split-operator by steps, split-operator per
 * element, independent per element) with an optional space-charge operator.
 * ------------------------------------------------------------------- */
enum { SB2_STEPPER_SPLIT_OPERATOR = 0, SB2_STEPPER_SPLIT_OPERATOR_ELEMENTS = 1,
       SB2_STEPPER_INDEPENDENT_ELEMENTS = 2 };

typedef struct sb2_propagator sb2_propagator;
/* sc may be NULL (Dummy_CO_options: no collective operator).  The lattice is
 * copied; its element attributes are read at creation. */
sb2_status sb2_propagator_create(const sb2_lattice* lattice, int32_t stepper, int32_t num_steps,
                                 const sb2_sc3d_options* sc, sb2_propagator** out);
sb2_status sb2_propagator_destroy(sb2_propagator* p);
sb2_status sb2_propagator_num_steps(sb2_propagator* p, int32_t* n);
/* Slices of independent operator `op` (0 = first half, 1 = second half) of
 * step `step`: triples (element index, left, right); returns the count in
 * *n (at most cap). */
sb2_status sb2_propagator_step_slices(sb2_propagator* p, int32_t step, int32_t op, double* out,
                                      int32_t cap, int32_t* n);
/* Propagator::propagate(sim, logger, turns) for one bunch, on `stream`
 * (cudaStream_t or NULL); returns after the device work is complete. */
sb2_status sb2_propagator_propagate(sb2_propagator* p, sb2_bunch* b, int32_t turns, void* stream);
/* Same over `count` consecutive steps starting at step `first` (steps wrap
 * around the turn). */
sb2_status sb2_propagator_propagate_steps(sb2_propagator* p, sb2_bunch* b, int32_t first,
                                          int32_t count, void* stream);
/* Replay each turn from a CUDA graph: the first turn with a given launch
 * signature is captured, later turns whose host-side re-derivation (op
 * lists, time steps, working-copy buffers) gives the same signature are
 * replayed with one graph launch.  propagate replays every turn;
 * propagate_steps launches the steps of its range that fall in one turn as
 * one graph (whole turns, and the partial turns at either end).  Off (0)
 * drops the cached graphs. */
sb2_status sb2_propagator_set_graphs(sb2_propagator* p, int32_t on);
/* With CUDA-graph turns on: capture, without running anything on the GPU,
 * the graphs that sb2_propagator_propagate_steps(p, b, first, count, ...)
 * will replay, so that call starts no capture.  The bunch is left as it was
 * (the steps are re-derived on the host only).  Does nothing with graphs
 * off, or for a bunch that has not been propagated yet (its first call
 * captures). */
sb2_status sb2_propagator_prepare_steps(sb2_propagator* p, sb2_bunch* b, int32_t first, int32_t count,
                                        void* stream);
sb2_status sb2_propagator_graph_stats(sb2_propagator* p, int64_t* captures, int64_t* replays);
/* Charge lost on lattice element `index` through the aperture operations
 * (Lattice_element::deposit_charge, aperture_operation.h:14-24), summed over
 * all bunches this propagator has propagated. */
sb2_status sb2_propagator_deposited_charge(sb2_propagator* p, int32_t index, double* charge);
/* Last space-charge solve: domain (left, h), rho, phi and the three field
 * components on the (gz, gy, gx) grid, scalars {fn_norm, factor, mean_std[6]}.
 * Any output may be NULL. */
sb2_status sb2_propagator_sc_last(sb2_propagator* p, double left[3], double h[3], double* rho,
                                  double* phi, double* ex, double* ey, double* ez, double scalars[8]);

/* A bunch split over several processes by particle range (one shard per
 * rank, each rank with its own propagator and bunch; the reference runs this
 * over MPI).  The library calls fn(ctx, data, count, on_host) wherever the
 * ranks exchange: the six moment sums of the adaptive domain and the
 * discard counts of update_total_num at each bookkeeping point
 * (core_diagnostics.cc:444, bunch.h:363-370), and the charge density after
 * every deposit (space_charge_3d_open_hockney.cc:572).  fn sums the `count`
 * doubles at `data` in place over the ranks and returns 0; every rank makes
 * the same calls in the same order.  on_host != 0: data is pinned host
 * memory (a host-side collective: gloo, MPI), and the library's work on its
 * stream is finished before each call; 0: data is device memory (NCCL), the
 * call comes without a host synchronisation, and fn must order its
 * collective after the work already queued on sb2_allreduce_stream() and
 * before the work queued there after fn returns (e.g. ncclAllReduce on that
 * stream).
 * The bunch's n_total and real_num are then the totals over the ranks (pass
 * the global real_num to every shard).  CUDA-graph turns and per-turn
 * diagnostics are not available on a sharded propagator.  fn = NULL
 * returns to a whole bunch. */
typedef int32_t (*sb2_allreduce_fn)(void* ctx, double* data, int64_t count, int32_t on_host);
sb2_status sb2_propagator_set_allreduce(sb2_propagator* p, sb2_allreduce_fn fn, void* ctx, int32_t on_host);
/* Typed sum-allreduce, the MPI_Allreduce(MPI_SUM) of the reference with its
 * datatype: dtype 0 = double, 1 = float; on_host as above.  With a typed
 * callback a mixed-precision propagator exchanges its FP32 charge grid as
 * float (half the bytes of the FP64 grid); the domain moments and valid
 * counts stay double.  Replaces the untyped callback (and is replaced by
 * it); fn = NULL returns to a whole bunch. */
typedef int32_t (*sb2_allreduce_typed_fn)(void* ctx, void* data, int64_t count, int32_t dtype, int32_t on_host);
sb2_status sb2_propagator_set_allreduce_typed(sb2_propagator* p, sb2_allreduce_typed_fn fn, void* ctx,
                                              int32_t on_host);
/* Inside a sum-allreduce callback: the cudaStream_t of the exchange (the
 * stream of the propagate call); NULL outside a callback. */
void* sb2_allreduce_stream(void);

/* Per-turn diagnostics on the device (Diagnostics_full2::do_update,
 * bunch/diagnostics_full2.cc:16-37): with capacity > 0 the propagator
 * appends one record for the initial state of its first propagate call and
 * one at the end of every turn, without host round trips (turn ends become
 * particle-pass boundaries).  A record is sb2_diagnostics_record_size()
 * doubles: num_particles, real_num, mean[6], std[6], min[3] and max[3] of
 * (x, y, cdt), mom2[36] (row major), corr[36], emitx, emity, emitz, emitxy,
 * emitxyz.  read copies up to max_records records (and the path length s
 * -- Reference_particle::get_s -- and turn count of each); capacity 0
 * disables. */
sb2_status sb2_propagator_set_diagnostics(sb2_propagator* p, int32_t capacity);
sb2_status sb2_propagator_read_diagnostics(sb2_propagator* p, int32_t max_records, int32_t* count, double* records,
                                           double* s, int32_t* turns);
int32_t sb2_diagnostics_record_size(void);

/* Lost-particle records (Diagnostics_loss, bunch.h:727-740,
 * diagnostics_loss.cc:6-34): with capacity > 0, every particle an aperture
 * discards is recorded on the device with its coordinates at that aperture.
 * read_losses returns up to max_records records of 10 doubles -- x, xp, y,
 * yp, cdt, dpop, id, and the repetition, s and s_n of the bunch reference at
 * the aperture -- ordered by aperture and id.  Not available with CUDA-graph
 * turns; capacity 0 disables. */
sb2_status sb2_propagator_set_loss_diagnostics(sb2_propagator* p, int32_t capacity);
sb2_status sb2_propagator_read_losses(sb2_propagator* p, int32_t max_records, int32_t* count, double* records);

/* Launch shape of the particle passes and the re-sort interval of the
 * cell-ordered working copy: the search space of the project's autotuner.
 * light_shape: light passes with 1 particle per thread and the next tile
 * prefetched (1), 2 per thread with (2) or without (0) prefetch, 1 per
 * thread with the next tile prefetched into shared memory by asynchronous
 * copies (3); full_occ:
 * passes with Yoshida integrators or bends at 2 (128 registers) or 3
 * (80 registers) CTAs per SM; full_ppt: particles per thread of the 2-CTA
 * variant (1, 2); quad_variant: passes whose only integrator is the
 * quadrupole Yoshida use the variant without the others, with one (1) or
 * two (2, at 2 CTAs per SM) particles per thread, or not (0);
 * ctas_per_sm: grid of the particle passes (1..12 x the SM count);
 * sort_interval: re-sort before every k-th space-charge kick; fft_plan: radix
 * plan of the FFT line passes (0: radix-8 passes first, 1: the radix-2/4
 * pass first, for lengths that are not powers of 8); deposit_chunk:
 * particles per thread of the tile deposit (4, 8; 0: warp groups with
 * global atomics).  The defaults
 * are the values measured best on the FODO workload of 4M macroparticles
 * (light_shape 3). */
typedef struct sb2_tune {
    int32_t light_shape, full_occ, full_ppt, quad_variant, ctas_per_sm, sort_interval;
    int32_t fft_plan, deposit_chunk;
} sb2_tune;
sb2_status sb2_propagator_get_tune(sb2_propagator* p, sb2_tune* out);
sb2_status sb2_propagator_set_tune(sb2_propagator* p, const sb2_tune* in);
/* Coordinate descent over the sb2_tune fields: every candidate propagates
 * `steps` untimed steps of a scratch copy of `b` (so the copy's cell order
 * has aged as in a long run), then `steps` more timed with CUDA events, and
 * the fastest is kept and applied.  The bunch, diagnostics, loss and step
 * records are left as they were.  trials (may be NULL) receives up to
 * max_trials rows of 7 doubles -- the six fields and the milliseconds --
 * and ntrials the number of trials run.  Not available on a sharded
 * propagator. */
sb2_status sb2_propagator_autotune(sb2_propagator* p, sb2_bunch* b, int32_t steps, sb2_tune* best, double* trials,
                                   int32_t max_trials, int32_t* ntrials);

/* Per-step counts (the bunch counts a diagnostics registered with
 * Bunch_simulator::reg_diag_per_step, bunch_simulator.h:230-238, sees at
 * every step end): with capacity > 0, the k-th step propagated after this
 * call writes record k -- n_valid (local_num), n_total and real_num after
 * the step's apertures -- into `host`.  The records are made on the device
 * by the pass bookkeeping, so the steps of one propagate call stay fused;
 * they are complete when the call returns.  Pinned (page-locked) `host`
 * memory is written by the device directly, at a device-side cursor, and
 * works with CUDA-graph turns; a pageable buffer gets stream-ordered copies
 * and is refused with graph turns.  step_counts_written gives the number of
 * records written; capacity 0 disables. */
typedef struct sb2_step_counts {
    int32_t n_valid;
    int32_t n_total;
    double real_num;
} sb2_step_counts;
sb2_status sb2_propagator_set_step_counts(sb2_propagator* p, sb2_step_counts* host, int32_t capacity);
sb2_status sb2_propagator_step_counts_written(sb2_propagator* p, int32_t* count);

/* ---------------------------------------------------------------------
 * Batch of independent jobs (no counterpart in the reference, which runs
 * bunch trains through one simulator): each job is a (propagator, bunch)
 * pair on its own CUDA stream; sb2_batch_run advances the listed slots by
 * the given number of turns concurrently and returns when all are done.
 * ------------------------------------------------------------------- */
typedef struct sb2_batch sb2_batch;
sb2_status sb2_batch_create(sb2_batch** out);
sb2_status sb2_batch_destroy(sb2_batch* q);
sb2_status sb2_batch_add(sb2_batch* q, sb2_propagator* p, sb2_bunch* b, int32_t* slot);
sb2_status sb2_batch_remove(sb2_batch* q, int32_t slot);
sb2_status sb2_batch_run(sb2_batch* q, const int32_t* slots, const int32_t* turns, int32_t n);
/* Asynchronous form for request loops: sb2_batch_launch enqueues `turns`
 * turns of one slot on its stream and returns at once (one launch in
 * flight per slot); sb2_batch_query sets *done to 1 once they have
 * finished -- bunch counters updated, device errors reported as the
 * status -- and to 0 while they run. */
sb2_status sb2_batch_launch(sb2_batch* q, int32_t slot, int32_t turns);
/* The listed slots advance `turns` turns in lockstep (one launch per kernel
 * kind per step for all of them): each job's step runs on the host as
 * usual, and its kernels go out as work-list launches over all listed
 * jobs -- the particle passes of every bunch in one launch per pass kernel,
 * the bookkeeping and domains in one, the charge deposits, Green functions,
 * convolutions and fields in one per grid shape.  Jobs need the same number
 * of steps per turn and the same launch sequence per step (one lattice with
 * different strengths; bunch sizes and grids may differ), otherwise
 * SB2_ERR_UNSUPPORTED; per-turn diagnostics, step-count records and
 * sharded propagators are not available, and every job needs its own
 * propagator and bunch.  Returns when the turns are done. */
sb2_status sb2_batch_run_lockstep(sb2_batch* q, const int32_t* slots, int32_t n, int32_t turns);
sb2_status sb2_batch_query(sb2_batch* q, int32_t slot, int32_t* done);

/* ---------------------------------------------------------------------
 * Collective operator alone: Space_charge_3d_open_hockney::apply_bunch
 * (space_charge_3d_open_hockney.cc:423-453).
 * ------------------------------------------------------------------- */
typedef struct sb2_sc3d sb2_sc3d;
sb2_status sb2_sc3d_create(const sb2_sc3d_options* opts, sb2_sc3d** out);
sb2_status sb2_sc3d_destroy(sb2_sc3d* sc);
/* One space-charge kick of the bunch over time_step [s]. */
sb2_status sb2_sc3d_apply(sb2_sc3d* sc, sb2_bunch* b, double time_step, void* stream);
/* Intermediate results of the last apply (as sb2_propagator_sc_last). */
sb2_status sb2_sc3d_last(sb2_sc3d* sc, double left[3], double h[3], double* rho, double* phi,
                         double* ex, double* ey, double* ez, double scalars[8]);

/* Space-charge kick that allocates nothing (no counterpart in the
 * reference): the same kick as sb2_sc3d_apply on caller-owned device arrays
 * (parts N x 7 column-major with column stride `stride`, masks N bytes;
 * parts updated in place), for callers that manage all device memory
 * themselves and cannot have the library call cudaMalloc/cudaFree.  All
 * workspaces live in one fixed 12 MiB device array that every GPU loading
 * the library holds until exit, so grids are limited to 65,536 cells with
 * doubled dimensions <= 128 (larger grids return SB2_ERR_INVALID).  The
 * first call on a device looks up that array's address and should come
 * before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race.  Returns after the stream is synchronised. */
sb2_status sb2_sc3d_apply_noalloc(const sb2_sc3d_options* opts, double* parts, int64_t stride,
                                  const uint8_t* masks, int64_t n, int32_t n_total, double real_num,
                                  int32_t charge, double mass, double value, int32_t kind, double time_step,
                                  void* stream);

/* ---------------------------------------------------------------------
 * Independent operations on explicit slices of a lattice.
 * ------------------------------------------------------------------- */
/* LibFF_operation over the given slices, in order: triples (element index,
 * left, right) of `lattice`; updates the bunch design reference particle
 * (initialised from the lattice reference particle on first use). */
sb2_status sb2_libff_apply(const sb2_lattice* lattice, const double* slices, int32_t nslices,
                           sb2_bunch* b, void* stream);
/* Aperture_operation<AP> for aperture type "finite", "circular",
 * "elliptical" or "rectangular" with the attributes of element `index`;
 * returns the number of discarded particles. */
sb2_status sb2_aperture_apply(const sb2_lattice* lattice, int32_t index, const char* aperture_type,
                              sb2_bunch* b, int32_t* ndiscarded, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SB2_H_ */
