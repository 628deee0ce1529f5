/* ising_b200.h — C ABI of the B200 Metropolis / parallel-tempering engine.
 *
 * Drop-in for the CPU sweep of EldosZhupanov/ising_engine (the "S1" path):
 * the 64-replica Metropolis sweep over CSR couplings, the dE / local-field
 * update and the DEO parallel-tempering replica exchange. Plain pointers and
 * sizes only; no C++ or torch types cross this boundary.
 *
 * Conventions
 *  - Every call returns an ie_status; no exception or abort crosses the ABI.
 *    After a non-zero status, ie_last_error() returns a message for the thread.
 *  - The caller owns every host buffer; the library copies what it needs and
 *    owns all device memory. A handle is not thread-safe; one CUDA stream per
 *    handle.
 *  - Spin words use the reference's init-word layout (ultimate.rs:272-275):
 *    bit r of word [cell][site] is replica r, cell = t + num_temps * p.
 *  - Integer mode (all linear terms and couplings integral, |value| <= 127 per
 *    coupling, local fields bounded by 127) is bit-exact with the reference for
 *    spins, energies, swap decisions and master-RNG position. Otherwise the f64
 *    mode runs the reference's f64 arithmetic in the reference's order.
 */
#ifndef ISING_B200_H
#define ISING_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IE_NUM_REPLICAS 64 /* NUM_REPLICAS, src/solver/types.rs:17 */

typedef enum ie_status {
    IE_OK = 0,
    IE_ERR_INVALID = 1,     /* bad shape, index out of range, bad config */
    IE_ERR_UNSUPPORTED = 2, /* e.g. num_slices != 1, more than 64 populations */
    IE_ERR_OOM = 3,         /* device allocation failed */
    IE_ERR_CUDA = 4,        /* CUDA runtime error */
    IE_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    IE_ERR_DEVICE = 6       /* device-side error word set (bounds check) */
} ie_status;

/* Mirrors QuboModel + CsrMatrix (src/core/hubo.rs:165-173,
 * src/core/csr_matrix.rs:6-10): both triangles stored, usize -> uint64. */
typedef struct ie_problem {
    uint64_t num_vars;
    const double* linear;        /* [num_vars] */
    const uint64_t* row_offsets; /* [num_vars + 1] */
    const uint64_t* col_indices; /* [nnz] */
    const double* values;        /* [nnz] */
    double energy_offset;
} ie_problem;

/* Mirrors the UltimateSolver fields the PT path reads (ultimate.rs:18-57).
 * exchange_interval is an extension: phase 2 of engine::step runs after every
 * k-th step (k = 1, the default when 0 is passed, is the reference). */
typedef struct ie_config {
    double temp_max;
    double temp_min;
    uint64_t sweeps_per_exchange;
    uint64_t total_exchanges;
    uint64_t seed;
    uint32_t num_temps;  /* default 10 (ultimate.rs:75) */
    uint32_t num_pops;   /* 1: PT; > 1: population annealing (ie_run_pa), cells t + num_temps * p */
    uint32_t num_slices; /* must be 1 (the Trotter branch is not on this path) */
    uint32_t exchange_interval;
    int32_t force_f64;   /* nonzero: use the f64 mode even for integral input */
    int32_t device;      /* CUDA device ordinal */
    int32_t pt_path;     /* 0: chosen by size; 1: one CTA runs all cells of the instance;
                            2: every cell is its own work item of the batched kernels, the
                            exchange runs between their launches (same results);
                            3: as 2, but one launch (one CTA) per cell, one after another:
                            the plain per-temperature method (level kernel only) */
    int32_t use_icm;     /* UltimateSolver::use_icm: an ICM sweep (src/solver/icm.rs) after every
                            exchange block of ie_run_pt; 0 by default */
    int32_t kernel_form; /* 0: integer-mode cells run on the level kernel (generator and
                            decision phases, all cells of the ladder in flight); 1: the
                            per-lane kernels only (same results) */
    uint32_t max_cluster; /* level kernel: most CTAs (a thread block cluster) running one
                             large cell, 1, 2, 4, 8 or 16; 0: chosen by size (at most 16) */
    int32_t bit_sliced;   /* level kernel, +-J problems (one coupling magnitude, lin = -sum w / 2,
                             degree <= 8): 0 the bit-sliced form (one thread per site for all 64
                             replicas) for problems too large for one CTA's shared memory and for
                             runs of at least one such cell per SM; 1 always; -1 never. Same
                             results either way */
} ie_config;

typedef struct ie_handle ie_handle;
typedef struct ie_batch ie_batch;

/* The population-annealing knobs of UltimateSolver (ultimate.rs:29-52). */
typedef struct ie_pa_config {
    double ess_threshold;              /* resample when ESS < ess_threshold * R; 0.5 by default
                                          (above 1: every stage after the first) */
    uint32_t ladder_tuning_iters;      /* 8 by default; 0 keeps the geometric ladder */
    uint32_t ladder_tuning_steps;      /* 10 by default */
    uint32_t post_resample_relaxation; /* 5 by default */
    int32_t ladder_mode;               /* 0: LadderMode::AcceptanceUniform (the default);
                                          1: LadderMode::FeedbackOptimized (round-trip tracking) */
    int32_t use_icm;                   /* ICM sweep after every stage (ultimate.rs:800-808); 0 by default */
} ie_pa_config;

/* PaDiagnostics (population_annealing.rs:34-45) plus the frozen ladder
 * shape. The arrays are caller-owned and may be NULL; `capacity` entries are
 * written at most, the counts are always complete. */
typedef struct ie_pa_report {
    double free_energy;
    uint64_t resample_events;
    uint64_t n_ess;          /* total_exchanges - 1 stages record an ESS */
    double* ess_history;     /* [capacity] */
    double* family_rho;      /* [capacity], one per resampling event */
    uint64_t* family_count;  /* [capacity] */
    uint64_t capacity;
    double* alphas;          /* [num_temps] or NULL */
} ie_pa_report;

const char* ie_last_error(void);
int ie_abi_version(void);

/* ---- single instance (engine::step seam and the UltimateSolver PT loop) ---- */

/* Replaces QuantumField::new + StepScratch::for_field + ChaCha8Rng::seed_from_u64
 * (ultimate.rs:152,235,299). Copies the problem to the device. */
ie_status ie_create(const ie_problem* problem, const ie_config* config, ie_handle** out);
ie_status ie_destroy(ie_handle* h);

/* is_clamped/clamp_val [num_vars] (engine.rs:567-571, ultimate.rs:154-159).
 * Call before ie_init_random. NULL clears all clamps. */
ie_status ie_set_clamps(ie_handle* h, const uint8_t* is_clamped, const int8_t* clamp_val);

/* ultimate.rs:248-290: one gen::<u64>() word per (t, v) from the master stream
 * (clamped sites take their value and draw nothing), then
 * calculate_replica_energies for every cell. */
ie_status ie_init_random(ie_handle* h);

/* UltimateSolver::with_gnn_heuristic (ultimate.rs:121-124, 256-263): from now
 * on the initial state (ie_init_random, and the fields ie_run_pa initializes)
 * is drawn per replica: replica r of an unclamped site v is one when its
 * gen_range(0.0..1.0) draw is below probs[v] (64 draws per cell and site);
 * probs [num_vars] is copied; NULL restores the random init. */
ie_status ie_set_init_probs(ie_handle* h, const double* probs);
/* The same initial words on the host (reference layout, bit r = replica r)
 * for `cells` cells from ChaCha8Rng::seed_from_u64(seed) after draw_offset
 * draws; *draws = the position after them. */
ie_status ie_warm_start_words(uint64_t seed, uint64_t draw_offset, const double* probs, const uint8_t* is_clamped,
                              const int8_t* clamp_val, uint64_t n, uint64_t cells, uint64_t* words, uint64_t* draws);

/* Sets spin words [num_temps * num_pops][num_vars] (cell t + num_temps * p)
 * directly (no master-stream draws) and recomputes the tracked energies. */
ie_status ie_set_spins(ie_handle* h, const uint64_t* words);

/* engine::step (engine.rs:573-819) n_steps times with a constant temperature
 * ladder temps[num_temps] (every population's ladder): base_seed draw,
 * index-order sweep of every cell, DEO exchange (every exchange_interval-th
 * step; population by population), phase toggle. Energies are re-synced
 * every 1000 steps as ultimate.rs:316-324 does (not on population handles,
 * whose driver re-syncs per stage). */
ie_status ie_step(ie_handle* h, const double* temps, uint32_t n_temps, uint64_t n_steps);

/* Per-step temperature schedule temps[n_steps][num_temps] (SA schedules). */
ie_status ie_run_schedule(ie_handle* h, const double* temps, uint32_t n_temps, uint64_t n_steps);

/* The UltimateSolver PT loop (ultimate.rs:234-336) with the geometric ladder
 * of the config: total_exchanges x sweeps_per_exchange steps, resync every
 * 1000 steps, the ICM sweep when use_icm, update_incumbent after every
 * exchange block (ultimate.rs:397-430). Requires ie_init_random (or
 * ie_set_spins) first; num_pops must be 1 (population handles run ie_run_pa). */
ie_status ie_run_pt(ie_handle* h);

ie_status ie_read_spins(ie_handle* h, uint64_t* words /* [num_temps * num_pops][num_vars] */);
ie_status ie_read_energies(ie_handle* h, double* energies /* [num_temps * num_pops][64] */);
/* swap attempts / accepts per adjacent pair [num_temps - 1] (engine.rs:545-551). */
ie_status ie_read_swap_stats(ie_handle* h, uint64_t* attempts, uint64_t* accepts);
/* Master-stream position (number of u64 draws so far) and DEO phase. */
ie_status ie_read_rng_state(ie_handle* h, uint64_t* draws, int32_t* deo_odd_phase);
/* Incumbent of ie_run_pt: energy (model energy incl. offset) and state [num_vars]. */
ie_status ie_read_incumbent(ie_handle* h, double* energy, int8_t* state);

/* Checkpoint of a handle's device state (handles with num_pops = 1): spin
 * words, replica energies, swap statistics, master-stream position, DEO
 * phase, steps run and the incumbent, as one blob. Loading it into a handle
 * created with the same problem and config continues the trajectory exactly
 * (the blob checks sites, cells, mode and its own spin digest).
 * The reference's replay anchor is the FNV-1a digest of the state
 * (src/engine_v2/state.rs:55-67); ie_state_digest is FNV-1a over the
 * little-endian bytes of the spin words in the reference layout (cell-major,
 * bit r = replica r), ie_fnv1a the same hash of any host buffer. */
ie_status ie_state_size(ie_handle* h, uint64_t* bytes);
ie_status ie_save_state(ie_handle* h, void* blob, uint64_t bytes);
ie_status ie_load_state(ie_handle* h, const void* blob, uint64_t bytes);
ie_status ie_state_digest(ie_handle* h, uint64_t* digest);
ie_status ie_fnv1a(const void* bytes, uint64_t n, uint64_t* digest);
/* Best replica of the final field in (t, r) order with strict < on the model
 * energy (ultimate.rs:345-368), merged with the incumbent (ultimate.rs:371-373). */
ie_status ie_read_best(ie_handle* h, double* energy, int8_t* state);
/* steepest_descent_1opt (src/solver/local_search.rs:19-57) on the device with
 * the handle's problem: polishes state [num_vars] (0/1) in place to a 1-opt
 * local minimum over the unclamped variables (is_clamped [num_vars] or NULL);
 * improvement = total energy decrease, as the reference returns it. */
ie_status ie_one_opt(ie_handle* h, int8_t* state, const uint8_t* is_clamped, double* improvement);

/* geometric ladder temps[i] = T_max * f^i, f = (T_min/T_max)^(1/(nt-1)),
 * computed with pow and powi exactly as ultimate.rs:238-246. */
ie_status ie_geometric_temps(double temp_max, double temp_min, uint32_t num_temps, double* out);
/* suggested_temp_range (src/solver/schedule.rs:21-43). */
ie_status ie_suggested_temp_range(const ie_problem* problem, double* temp_max, double* temp_min);

/* ---- batched: many single-cell SA instances in one persistent launch ---- */

typedef struct ie_batch_config {
    int32_t device;
    int32_t force_f64;
    uint32_t threads_per_block; /* level kernel: threads per CTA (multiple of 32, <= 256; 0: 256) */
    uint32_t blocks_per_sm;     /* cap on resident CTAs per SM per class, 0 = as many as fit */
    int32_t disable_windows;    /* nonzero: never use the windowed kernel for large instances */
    int32_t use_graph;          /* nonzero: ie_batch_run_schedule replays one CUDA graph holding
                                   the launches of every work class (captured on first use and
                                   again when the classes or the schedule length change) */
    int32_t kernel_form;        /* 0: the level kernel (default); 1: the per-lane kernels.
                                   Same spins; f64 energies are the FP64 recompute of the final
                                   state on the level kernel, the tracked sum on the others */
    uint32_t item_sites;        /* level kernel: spin words per CTA work item (0: 4096) */
    uint32_t tie_shift;         /* test hook, 0 in normal use: level-kernel decisions compare only
                                   the top 32 - tie_shift bits of the stored outputs, so the exact
                                   path (outputs recomputed from the lane seed) runs often */
    int32_t bit_sliced;         /* as ie_config::bit_sliced */
    int32_t bulk_ring;          /* per-lane kernels (kernel_form 1): nonzero streams the site-record
                                   chunks by 1D bulk copies completing on mbarriers instead of
                                   16-byte cp.async copies (same results; cp.async is the default,
                                   measured faster on these kernels) */
} ie_batch_config;

/* count problems, each run as one cell of 64 replicas with its own seed. */
ie_status ie_batch_create(const ie_problem* problems, uint32_t count, const uint64_t* seeds,
                          const ie_batch_config* config, ie_batch** out);
ie_status ie_batch_destroy(ie_batch* b);
/* Random init of every instance (ultimate.rs:248-290 with num_temps = 1). */
ie_status ie_batch_init_random(ie_batch* b);
/* Runs temps[n_steps] (one temperature per step, shared by all instances) on
 * every instance: engine::step with num_temps = 1, resync every 1000 steps. */
ie_status ie_batch_run_schedule(ie_batch* b, const double* temps, uint64_t n_steps);
/* Same schedule, one launch per instance in sequence (the plain method). */
ie_status ie_batch_run_schedule_plain(ie_batch* b, const double* temps, uint64_t n_steps,
                                      uint32_t first, uint32_t count);
/* Autotuner: times trial_steps of the schedule temps[] for a grid of launch
 * shapes, restoring the device state after every trial, and keeps the fastest.
 * Level kernel (kernel_form 0): spin words per CTA work item in {1024, 2048,
 * 4096, 8192} x threads per CTA in {128, 256}; chosen[4] (may be NULL)
 * receives {item_sites, threads, 0, 0}. Per-lane kernels: the thread-class
 * thresholds (instances above a size threshold get 2 or 4 threads per
 * generator lane); chosen receives {n4_int, n2_int, n4_f64, n2_f64}. */
ie_status ie_batch_autotune(ie_batch* b, const double* temps, uint64_t trial_steps, uint32_t* chosen);
/* Spin words of instance i at words + offsets[i] (offsets = prefix sums of n). */
ie_status ie_batch_read_spins(ie_batch* b, uint64_t* words);
ie_status ie_batch_read_energies(ie_batch* b, double* energies /* [count][64] */);
ie_status ie_batch_read_draws(ie_batch* b, uint64_t* draws /* [count] */);
/* FP64 recompute of every instance's energies on the device, reference order. */
ie_status ie_batch_recompute_energies(ie_batch* b, double* energies /* [count][64] */);
/* Device time of the last run call in milliseconds (CUDA events on its stream). */
ie_status ie_batch_last_run_ms(ie_batch* b, double* ms);
/* Work classes of the last batched run: for class k < min(max_classes, *n_classes),
 * info[5k..5k+4] = {mode (0 integer, 1 f64, 2 the level kernel's bit-sliced +-J form),
 * threads per lane (8 = windowed kernel, 16 = chain kernel, 32 = level kernel),
 * shared-memory spin capacity, work items, valid}, ms[k] = its device time. */
ie_status ie_batch_class_report(ie_batch* b, uint32_t max_classes, uint32_t* n_classes, uint32_t* info,
                                double* ms);
/* Number of kernel launches the last run call issued. */
ie_status ie_batch_last_launches(ie_batch* b, uint64_t* launches);
/* Level kernel: number of decisions taken on its exact path (output
 * recomputed from the lane seed) since the batch was created. */
ie_status ie_batch_exact_decisions(ie_batch* b, uint64_t* count);

/* Coefficients of x^steps mod P(x), P the characteristic polynomial of the
 * Xoshiro256 state transition (engine.rs:115-121): bit i of out[i / 64] is the
 * coefficient of x^i. The state after `steps` more steps is the XOR of the
 * states after i steps over the set coefficients i < 256 (the jump the level
 * kernel uses to start a lane's stream mid-sweep). out: [4]. */
ie_status ie_xoshiro_jump_poly(uint64_t steps, uint64_t* out);

/* ---- one SA run with no device allocation (no reference counterpart) ----
 * For callers that cannot allocate device memory: hosts whose framework owns
 * a fixed device pool and forbids other allocators, and services that must
 * not block or fail on an allocation mid-request. The problem and the outputs are in device memory the
 * caller already owns; all scratch lives in one file-scope device array of
 * 12 MiB that every GPU loading this library holds until process exit.
 * Limits: num_vars <= 16384, nnz <= 262144 (both triangles), n_steps <= 65536;
 * larger inputs return IE_ERR_INVALID. The first call on a device looks up the
 * array's device address (kept for the life of that device's CUDA context);
 * make that first call before any stream capture. The caller's current device
 * is restored before the call returns. Calls share the array, so calls that
 * overlap on the GPU (other threads or streams) race; serialize them. The run
 * is the f64 mode of the batched sweep (same spins and energies as
 * ie_batch_run_schedule for the same problem, seed and temperatures); it
 * returns after the stream has finished the run. */
typedef struct ie_problem_device {
    uint32_t num_vars;
    uint32_t nnz;
    const uint32_t* row_offsets; /* device, [num_vars + 1] */
    const uint32_t* col_indices; /* device, [nnz] */
    const double* values;        /* device, [nnz] */
    const double* linear;        /* device, [num_vars] */
} ie_problem_device;

/* temps: host [n_steps]; words: device [num_vars] (bit r = replica r);
 * energies: device [64]; stream: a cudaStream_t or NULL. */
ie_status ie_sa_run_static(const ie_problem_device* problem, uint64_t seed, const double* temps,
                           uint64_t n_steps, uint64_t* words, double* energies, int32_t device,
                           void* stream);

/* ---- serving: continuous batching of SA requests ----
 * Replaces the request loop of the reference's HTTP server
 * (src/bin/server_api.rs:180-213: validate, take a compute permit, solve on the
 * Rayon pool, return) with a device-resident request pool. Requests are
 * single-cell SA solves (64 replicas, one temperature per step). A request
 * is admitted, first come first served, once a slot and room in every device
 * pool (sites, couplings, records, schedule) are free; it stays resident
 * (spins, energies, generator position) until its schedule is done, and
 * every tick advances each resident request in one group of persistent
 * launches, so requests of different sizes and arrival times share the GPU.
 * On the level kernel a tick gives each request the steps that its work item
 * runs in about tick_us of device time, from the cycles per step that item
 * measured in the previous tick (a request's first tick: at most 64 steps);
 * on the per-lane kernels up to max(1, site_budget / N) steps. A request's result does not depend on
 * what else is resident: it equals ie_batch_run_schedule of the same problem,
 * seed and temperatures alone.
 * ie_serve_submit, ie_serve_poll and ie_serve_result may be called from any
 * thread, also while ie_serve_tick runs; ie_serve_tick from one thread at a
 * time. */
typedef struct ie_serve ie_serve;
typedef struct ie_serve_config {
    int32_t device;
    int32_t force_f64;
    uint32_t max_requests;       /* resident request slots (0: 4096) */
    uint32_t site_budget;        /* site-steps per request per tick (0: 65536) */
    uint64_t max_sites;          /* summed num_vars of resident requests (0: 2^24) */
    uint64_t max_couplings;      /* summed stored couplings, both triangles (0: 2^27) */
    uint64_t max_schedule_steps; /* summed schedule lengths (0: 2^25) */
    int32_t kernel_form;         /* 0: the level kernel (default); 1: the per-lane kernels */
    uint32_t tick_us;            /* level kernel: device time per tick to plan for, microseconds
                                    (0: 200000) */
} ie_serve_config;

ie_status ie_serve_create(const ie_serve_config* config, ie_serve** out);
ie_status ie_serve_destroy(ie_serve* s);
/* Validates and prepares the request on the calling thread and queues it.
 * temps: host [n_steps]; is_clamped / clamp_val: [num_vars] or NULL.
 * IE_ERR_OOM when the request alone exceeds a pool's capacity,
 * IE_ERR_UNSUPPORTED when it does not fit the kernels' shared memory. */
ie_status ie_serve_submit(ie_serve* s, const ie_problem* problem, uint64_t seed, const double* temps,
                          uint64_t n_steps, const uint8_t* is_clamped, const int8_t* clamp_val, uint64_t* id);
/* Admits queued requests, runs one tick, retires finished requests. */
ie_status ie_serve_tick(ie_serve* s, uint32_t* n_active, uint32_t* n_pending, uint32_t* n_finished);
/* Ids of finished requests whose results have not been taken yet. */
ie_status ie_serve_poll(ie_serve* s, uint64_t* ids, uint32_t max_ids, uint32_t* n_ids);
/* Takes a finished request's result: words [num_vars] (bit r = replica r) and
 * energies [64] (model energy without the offset); frees its record. */
ie_status ie_serve_result(ie_serve* s, uint64_t id, uint64_t* words, double* energies);
/* Device bytes a request would hold while resident (its admission footprint). */
ie_status ie_serve_footprint(ie_serve* s, const ie_problem* problem, uint64_t n_steps, uint64_t* bytes);
/* Device time of the last tick and kernel launches in it. */
ie_status ie_serve_last_tick(ie_serve* s, double* ms, uint64_t* launches);

/* ---- engine_v2 (S2) bit-sliced state and operators ----
 * The integral-couplings state backend SparseBitSlice
 * (src/engine_v2/backends/sparse_bitslice.rs:19-346) on the device, driven at
 * the granularity of one operator application: MetropolisSweep::apply
 * (src/engine_v2/operators/metropolis_sweep.rs:95-146) and
 * ReplicaExchange::apply (src/engine_v2/operators/replica_exchange.rs:61-110).
 * The per-site delta_e_into / apply_flips of the SpinState trait
 * (src/engine_v2/state.rs:70-148) are too fine for a device call and are not
 * exported. `ir` is a ProblemIR (src/engine_v2/ir.rs:14-69): both triangles,
 * rows sorted, duplicates merged, no zero weights, integral values.
 * The operator's ChaCha8Rng is ChaCha8Rng::seed_from_u64(seed) after
 * `draw_offset` 64-bit draws; a Metropolis call consumes sweeps * n * r
 * draws (a Gibbs call as many), an exchange call one per attempted pair
 * (*proposed). */
typedef struct ie_v2 ie_v2;
/* init: [num_vars] 0/1, copied into every replica (SparseBitSlice::new). */
ie_status ie_v2_create(const ie_problem* ir, uint32_t num_replicas, const uint8_t* init, int32_t device,
                       ie_v2** out);
ie_status ie_v2_destroy(ie_v2* h);
/* temps: per-replica temperatures, replica k uses temps[k % n_temps]. */
ie_status ie_v2_metropolis(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t sweeps, uint64_t seed,
                           uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted);
ie_status ie_v2_exchange(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t rounds, uint64_t seed,
                         uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted);
/* GibbsColorSweep::apply (src/engine_v2/operators/gibbs_color_sweep.rs:119-165):
 * heat-bath resampling in chromatic order, sweeps * n * r draws; a temperature
 * <= 0 (or NaN) is the greedy limit, as in the reference. */
ie_status ie_v2_gibbs(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t sweeps, uint64_t seed,
                      uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted);
/* planes: [num_vars * ceil(r / 64)] (bit b of word q of a site = replica 64q + b);
 * energies: [r] from the ledger (either may be NULL). */
ie_status ie_v2_read(ie_v2* h, uint64_t* planes, double* energies);
/* SpinState::audit: largest |ledger - recomputed| energy; 0 on an exact state. */
ie_status ie_v2_audit(ie_v2* h, double* drift);
/* ProblemIR::greedy_coloring (src/engine_v2/ir.rs:114-139), host only. */
ie_status ie_v2_coloring(const ie_problem* ir, uint32_t* colors);

/* ---- population annealing with PT equilibration (num_pops > 1) ----
 * UltimateSolver::solve_population_annealing_diag (ultimate.rs:576-852) on a
 * handle created with num_pops > 1, entered as solve_with_pa_diagnostics does
 * (ultimate.rs:858-890: clamps from ie_set_clamps, no presolve): ladder
 * tuning on a throwaway field, then total_exchanges annealing stages of
 * sweeps_per_exchange engine::step calls over all populations, Boltzmann
 * reweighting at the cold level, systematic resampling with shuffled
 * offspring when the ESS falls below the threshold, post-resampling
 * relaxation, an exact energy re-sync and the incumbent after every stage.
 * The handle's master stream must be fresh (ChaCha8Rng::seed_from_u64(seed)).
 * Afterwards ie_read_best / ie_one_opt finish the solve (ultimate.rs:806-845). */
ie_status ie_run_pa(ie_handle* h, const ie_pa_config* config, ie_pa_report* report);

/* population_annealing.rs primitives (host only). */
ie_status ie_pa_normalized_weights(const double* log_w, uint64_t r, double* w_out);
ie_status ie_pa_effective_sample_size(const double* w, uint64_t r, double* ess);
ie_status ie_pa_free_energy_increment(const double* log_w, uint64_t r, double* out);
/* families are summed in ascending id order */
ie_status ie_pa_family_entropy(const uint64_t* family_ids, uint64_t r, double* rho, uint64_t* families);
ie_status ie_pa_systematic_resample(const double* w, uint64_t r, double u, uint64_t* counts);
ie_status ie_pa_adapt_spacings(const double* spacings, const double* acceptance, uint64_t k, double* out);
ie_status ie_pa_feedback_optimized_alphas(const double* alphas, const double* flow, uint64_t nt, double damping,
                                          double* out);

/* ---- finishers after the anneal (host only) ----
 * steepest_descent_2opt_escapes (src/solver/local_search.rs:123-143): 1-opt
 * descent, then the steepest improving 2-flip along the coupling graph's
 * edges, repeated until neither improves; free variables only (is_clamped may
 * be NULL). state [num_vars] 0/1 is polished in place; *improvement (may be
 * NULL) = max(0, E_before - E_after). */
ie_status ie_two_opt(const ie_problem* problem, int8_t* state, const uint8_t* is_clamped, double* improvement);
/* The path-relinking finisher (ultimate.rs:436-479, src/solver/elite.rs):
 * the current state and every replica of words [cells][num_vars] (the layout
 * ie_read_spins returns: bit r = replica r) feed an elite archive (8 entries,
 * Hamming radius max(num_vars / 10, 1)); every pair of elites is relinked
 * greedily and polished by 1-opt; the best state (strictly better than the
 * current one, else the current one) is written back to `state`, its model
 * energy to *energy (may be NULL). Host only. */
ie_status ie_path_relink(const ie_problem* problem, const uint64_t* words, uint64_t cells,
                         const uint8_t* is_clamped, int8_t* state, double* energy);

/* ---- presolve and decomposition (host only) ----
 * full_presolve (src/presolve/mod.rs:279-324): roof-duality strong
 * persistencies (src/presolve/qpbo.rs) of the clamp-reduced model unioned
 * with probing weak persistencies; writes the fixings beyond the user's
 * clamps (out_idx / out_val: [num_vars] capacity, may be NULL to count). */
ie_status ie_presolve(const ie_problem* problem, const uint64_t* clamp_idx, const int8_t* clamp_val,
                      uint64_t n_clamps, uint64_t* out_idx, int8_t* out_val, uint64_t* n_out);
/* connected_components (mod.rs:189-218) of the graph of nonzero couplings
 * among active variables: component[v] = its component (numbered by
 * smallest vertex) or UINT64_MAX for inactive v. */
ie_status ie_connected_components(const ie_problem* problem, const uint8_t* active, uint64_t* component,
                                  uint64_t* n_components);

/* ---- measurement helper (no reference counterpart) ----
 * Measured roofline denominators on `device`: int32 LOP3/IADD3 throughput
 * (ops/s) and Xoshiro256++ step+compare throughput (outputs/s), the per-attempt
 * work the bit-exact sweep cannot avoid. */
ie_status ie_probe_peaks(int32_t device, double* int_ops_per_s, double* xoshiro_per_s);

#ifdef __cplusplus
}
#endif

#endif /* ISING_B200_H */
