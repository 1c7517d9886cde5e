/*
 * wlg.h — C-ABI of the B200 replica-exchange Wang–Landau (REWL) walker engine.
 *
 * The reference sampler (Faikert/replica_exchange_wang_landau, C++20) has no FFI layer;
 * its drop-in seam is the C++ function
 *
 *     RewlResult run_rewl(const ParallelContext&, std::shared_ptr<const Couplings>,
 *                         const RunConfig&);                 (include/wl/parallel.hpp:35-36)
 *
 * plus the physics helpers it is built from (include/wl/physics.hpp:37-84) and the
 * per-walker API its tests drive (include/wl/wang_landau.hpp:91-175).  Every entry point
 * below names the reference interface it replaces.  Conventions:
 *   - every function returns a wlg_status (0 = ok); the message of the last failure on the
 *     calling thread is returned by wlg_last_error();
 *   - the engine owns all device memory; the caller owns every host buffer it passes;
 *   - an engine is used from one host thread at a time;
 *   - array arguments are plain host pointers with sizes; no torch or CUDA types appear.
 */
#ifndef WLG_H
#define WLG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WLG_ABI_VERSION 1

typedef enum wlg_status {
    WLG_OK = 0,
    WLG_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference            */
    WLG_ERR_INIT_FAILED = 2,      /* walker initialisation failed (std::runtime_error)  */
    WLG_ERR_ESCAPED = 3,          /* "Walker escaped its energy window"                 */
    WLG_ERR_DEVICE = 4,           /* CUDA error, or no usable sm_100 device             */
    WLG_ERR_TIMEOUT = 5,          /* a bounded device wait gave up                      */
    WLG_ERR_RUNTIME = 6,          /* other std::runtime_error conditions                */
    WLG_ERR_LOGIC = 7,            /* std::logic_error                                   */
    WLG_ERR_OUT_OF_RANGE = 8,     /* std::out_of_range                                  */
    WLG_ERR_IO = 9                /* file could not be read or written                  */
} wlg_status;

typedef enum wlg_precision {
    WLG_PRECISION_FP64 = 0, /* J in FP64: bit-exact with the reference                  */
    WLG_PRECISION_FP32 = 1, /* J in FP32, FP64 fields, periodic FP64 recompute          */
    WLG_PRECISION_BF16 = 2  /* J in BF16 with a per-row FP32 scale, FP64 fields         */
} wlg_precision;

typedef enum wlg_stage { /* wl::RefinementStage (include/wl/wang_landau.hpp:58) */
    WLG_STAGE_WANG_LANDAU = 0,
    WLG_STAGE_INVERSE_TIME = 1,
    WLG_STAGE_FROZEN = 2
} wlg_stage;

/* A dipolar Ising system: wl::Geometry + coupling scale + cutoff
 * (include/wl/physics.hpp:13-35; apps/wl_run.cpp:81-83 selects CSR when cutoff > 0). */
typedef struct wlg_system {
    uint64_t n;               /* number of sites                                       */
    const double* positions;  /* n x 3 (x, y, z), row-major                            */
    const double* axes;       /* n x 3 unit easy axes                                  */
    double box[3];            /* box lengths; a zero length leaves that axis open      */
    int32_t periodic;         /* minimum image on the positive-length axes             */
    double coupling_scale;    /* D                                                     */
    double cutoff;            /* > 0 selects the CSR backend with |r| <= cutoff         */
} wlg_system;

/* Prebuilt couplings: the J of a wl::Couplings object (include/wl/physics.hpp:41-49) as
 * Couplings::at(i, j) exports it, for callers that hold couplings rather than a geometry
 * (run_rewl takes std::shared_ptr<const Couplings>, include/wl/parallel.hpp:35-36).  Dense
 * (DenseCouplings, src/physics.cpp:172-188): `dense` is the n x n row-major matrix and the CSR
 * members are unused.  CSR (CsrCouplings, src/physics.cpp:197-229): `dense` is NULL and
 * row_offsets[n+1] / columns[nnz] / values[nnz] hold each row's stored couplings by ascending
 * column.  Either form must be symmetric with a zero diagonal and finite values, as both
 * reference backends are; otherwise creation fails with WLG_ERR_INVALID_ARGUMENT. */
typedef struct wlg_couplings {
    uint64_t n;                  /* number of sites                                        */
    const double* dense;         /* n x n, or NULL for the CSR form                        */
    uint64_t nnz;                /* CSR: stored couplings                                  */
    const uint64_t* row_offsets; /* CSR: n + 1 offsets into columns / values               */
    const uint64_t* columns;     /* CSR: column of each stored coupling                    */
    const double* values;        /* CSR: value of each stored coupling                     */
} wlg_couplings;

/* wl::WlParameters (include/wl/wang_landau.hpp:40-56), field for field. */
typedef struct wlg_wl_parameters {
    double flatness;
    uint64_t minimum_visits;
    double final_factor;
    uint64_t check_interval_attempts;
    uint64_t force_accept_after_attempts;
    int32_t inverse_time_enabled;
    uint64_t initialization_max_attempts;
    double initialization_target_fraction;
    double initialization_temperature_fraction;
    uint64_t initialization_stall_attempts_per_spin;
    double initialization_temperature_multiplier;
    double initialization_max_temperature_fraction;
    int32_t collect_window_statistics;
    double round_trip_margin_fraction;
    int32_t nalivaiko_mod;
} wlg_wl_parameters;

/* The part of wl::RunConfig that run_rewl reads (include/wl/io.hpp:12-58), with MCS
 * intervals already resolved to attempts (RunConfig::resolve_mcs, src/io.cpp:210-236). */
typedef struct wlg_run_config {
    double emin, emax, bin_width;           /* EnergyGrid                               */
    uint64_t windows;                       /* energy windows                           */
    uint64_t walkers_per_window;            /* RunConfig::walkers_per_rank              */
    double overlap;                         /* partition_windows overlap                */
    const uint64_t* explicit_windows;       /* NULL, or 2*windows (begin, end) bins     */
    uint64_t seed;
    wlg_wl_parameters wl;
    uint64_t exchange_interval_attempts;
    uint64_t max_attempts;                  /* 0 = run until every walker is frozen     */
    uint64_t checkpoint_interval_attempts;
    const char* checkpoint_path;            /* NULL/"" = none; used for 1 window x 1    */
    const int8_t* initial_spins;            /* NULL, or windows*walkers x n spins       */
    const uint8_t* initial_spins_present;   /* NULL = all present; else one per walker  */
    double progress_interval_seconds;       /* 0 disables the progress line             */
    int32_t coupling_precision;             /* wlg_precision                            */
    uint64_t recompute_interval_attempts;   /* FP32/BF16 only: FP64 field recompute     */
} wlg_run_config;

/* wl::HistogramStatistics (include/wl/wang_landau.hpp:60-67). */
typedef struct wlg_histogram_statistics {
    uint64_t active_bins;
    uint64_t covered_bins;
    uint64_t minimum;
    double mean;
    double min_over_mean;
    double coverage;
} wlg_histogram_statistics;

/* wl::WalkerStatistics (include/wl/io.hpp:60-75). */
typedef struct wlg_walker_statistics {
    uint64_t walker_id;
    uint64_t window_id;
    int32_t mpi_rank;
    uint64_t attempted;
    uint64_t accepted;
    uint64_t forced_accepted;
    uint64_t attempts_since_last_accepted;
    double energy;
    double factor;
    uint64_t active_bins;
    uint64_t minimum_histogram;
    double mean_histogram;
    double min_over_mean;
    uint64_t round_trips;
} wlg_walker_statistics;

/* The scalar part of wl::RewlResult (include/wl/parallel.hpp:23-31). */
typedef struct wlg_run_totals {
    uint64_t attempted;
    uint64_t accepted;
    uint64_t forced_accepted;
    uint64_t exchange_attempted;
    uint64_t exchange_accepted;
    int32_t converged;
    uint64_t epochs;
} wlg_run_totals;

/* Device timing of a run of epochs (no counterpart in the reference, which only reports
 * wall-clock time, apps/wl_run.cpp:175-178). */
typedef struct wlg_epoch_timing {
    uint64_t epochs;     /* epochs run                                                   */
    double walk_ms;      /* device time of the sweep kernels (CUDA events)               */
    double exchange_ms;  /* device time of the exchange kernels                          */
    double total_ms;     /* device time from the first launch to the last                */
    uint64_t attempted;  /* attempts made in these epochs, all walkers                   */
    uint64_t accepted;   /* accepted flips in these epochs, all walkers                  */
} wlg_epoch_timing;

/* Drift of a mixed-precision run (coupling_precision FP32 or BF16), accumulated over its
 * periodic FP64 recomputes (recompute_interval_attempts).  No counterpart in the reference,
 * which stores J in FP64 only. */
typedef struct wlg_precision_report {
    int32_t coupling_precision;  /* wlg_precision of the run                                  */
    int32_t pad;
    uint64_t recompute_interval_attempts; /* 0: no recompute scheduled                        */
    uint64_t recomputes;         /* FP64 recompute passes made                                */
    uint64_t resynced;           /* walker states replaced by the FP64 values                 */
    uint64_t deferred;           /* resyncs deferred because E64 fell outside the window     */
    uint64_t bin_changes;        /* resyncs that moved a walker's current bin                 */
    double max_field_drift;      /* max over recomputes, walkers, sites of |h - h64|          */
    double max_energy_drift;     /* max over recomputes and walkers of |E - E64|              */
} wlg_precision_report;

/* wl::WalkerSnapshot (include/wl/wang_landau.hpp:74-89).  The array members point to
 * caller-owned buffers: spins and fields hold n entries, log_g/histogram/active hold
 * grid-bins entries (the whole grid, as in the reference). */
typedef struct wlg_snapshot {
    uint64_t walker_id;
    int8_t* spins;
    double* fields;
    double energy;
    double* log_g;
    uint64_t* histogram;
    uint8_t* active;
    double factor;
    uint64_t attempted;
    uint64_t accepted;
    uint64_t forced_accepted;
    uint64_t last_accepted_attempt;
    uint8_t stage;
    uint64_t rng_state[4];
} wlg_snapshot;

typedef struct wlg_engine wlg_engine;

/* ---- library ------------------------------------------------------------------ */

/* Returns WLG_ABI_VERSION. */
int32_t wlg_abi_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* wlg_last_error(void);
/* Selects the CUDA device that engines created afterwards on this thread use (the
 * library carries its own CUDA runtime).  One process per GPU is the intended layout.  No
 * counterpart in the reference, which is CPU-only. */
wlg_status wlg_set_device(int32_t device);
/* Fills defaults equal to the reference's RunConfig/WlParameters member initialisers
 * (include/wl/io.hpp:12-58, include/wl/wang_landau.hpp:40-56) with MCS resolved for n
 * spins as RunConfig::resolve_mcs does (src/io.cpp:210-236). */
wlg_status wlg_default_run_config(uint64_t n, wlg_run_config* out);

/* ---- host-side helpers (no GPU needed) ---------------------------------------- */

/* EnergyGrid::bins / EnergyGrid::index (src/wang_landau.cpp:22-34).  *bin = -1 when the
 * reference returns std::nullopt. */
wlg_status wlg_grid_bins(double emin, double emax, double width, uint64_t* bins);
wlg_status wlg_grid_index(double emin, double emax, double width, double energy, int64_t* bin);
/* partition_windows (src/wang_landau.cpp:40-61); out holds 2*count (begin, end). */
wlg_status wlg_partition_windows(uint64_t bins, uint64_t count, double overlap, uint64_t* out);
/* Geometry::validate (src/physics.cpp:34-56). */
wlg_status wlg_validate_system(const wlg_system* system);
/* save_checkpoint / load_checkpoint: the WLCHKP3 binary format (src/io.cpp:539-572);
 * load also reads WLCHKP1/WLCHKP2.  For load, sizes are returned first when the array
 * pointers in *s are NULL (*n_spins, *n_bins set), then filled on a second call. */
wlg_status wlg_checkpoint_save(const char* path, const wlg_snapshot* s, uint64_t n_spins,
                               uint64_t n_bins);
wlg_status wlg_checkpoint_load(const char* path, wlg_snapshot* s, uint64_t* n_spins,
                               uint64_t* n_bins);

/* ---- physics on the device ---------------------------------------------------- */

/* DenseCouplings / CsrCouplings construction (src/physics.cpp:172-223), returned as the
 * dense n x n matrix that Couplings::at(i, j) reads (zeros off the CSR pattern).  With
 * precision FP32/BF16 the stored (rounded, row-scaled) values are returned as doubles. */
wlg_status wlg_couplings_dense(const wlg_system* system, int32_t precision, double* out);
/* CsrCouplings pattern (src/physics.cpp:197-223): row_offsets[n+1], columns[nnz],
 * values[nnz].  Call with columns == NULL to get *nnz first. */
wlg_status wlg_couplings_csr(const wlg_system* system, uint64_t* nnz, uint64_t* row_offsets,
                             uint64_t* columns, double* values);
/* local_fields + total_energy (src/physics.cpp:238-259) for `count` spin configurations
 * (count x n spins), computed with the reference's summation order. */
wlg_status wlg_local_fields(const wlg_system* system, const int8_t* spins, uint64_t count,
                            double* fields, double* energies);
/* The same results as wlg_local_fields for callers that cannot allocate device memory (a
 * host whose own pool already holds the GPU's memory, code that must not add the device
 * synchronisation cudaMalloc/cudaFree can cause, hosts that forbid allocation after
 * start-up).  No counterpart in the reference.  Nothing is allocated: the couplings and all
 * staging live in one static device array of 18 MiB that every GPU loading this library
 * keeps until the process exits.  Limits: dense systems only (cutoff 0), n <= 1024 sites,
 * count <= 65536 configurations and count * n <= 1048576; larger inputs return
 * WLG_ERR_INVALID_ARGUMENT with the limit in the message.  Every call looks up the array's
 * device address on the current device; the first call on a device loads the library's
 * device code and should come before any stream capture.  Work runs on the legacy default
 * stream, so no call may run while another thread holds a global-mode stream capture.
 * Calls share the array: calls that overlap on the GPU race. */
wlg_status wlg_local_fields_noalloc(const wlg_system* system, const int8_t* spins,
                                    uint64_t count, double* fields, double* energies);

/* ---- the REWL engine: run_rewl (src/parallel.cpp:276-747) ---------------------- */

/* Builds J, constructs windows*walkers walkers (WangLandauWalker ctor with target
 * Metropolis initialisation, src/wang_landau.cpp:63-242) and restores a checkpoint when
 * the reference would (src/parallel.cpp:354-360). */
wlg_status wlg_engine_create(const wlg_system* system, const wlg_run_config* config,
                             wlg_engine** engine);
/* The same engine from prebuilt couplings instead of a geometry: run_rewl's own inputs
 * (std::shared_ptr<const Couplings> + RunConfig, include/wl/parallel.hpp:35-36).  The dense
 * form runs the dense sweeps, the CSR form the CSR sweeps, exactly as an engine created from
 * the geometry those couplings came from. */
wlg_status wlg_engine_create_from_couplings(const wlg_couplings* couplings, const wlg_run_config* config,
                                            wlg_engine** engine);
void wlg_engine_destroy(wlg_engine* engine);
/* The epoch loop of run_rewl (src/parallel.cpp:376-534) until every walker is frozen or
 * the attempt limit is reached. */
wlg_status wlg_engine_run(wlg_engine* engine, wlg_run_totals* totals);
/* At most max_epochs epochs of the same loop; *done = 1 once the run has terminated. */
wlg_status wlg_engine_run_epochs(wlg_engine* engine, uint64_t max_epochs,
                                 uint64_t* epochs_run, int32_t* done);
wlg_status wlg_engine_totals(wlg_engine* engine, wlg_run_totals* totals);
/* The same epochs as wlg_engine_run_epochs, launched one kernel at a time with CUDA events
 * around each kernel on the engine's stream (profiling; no counterpart in the reference). */
wlg_status wlg_engine_time_epochs(wlg_engine* engine, uint64_t epochs, wlg_epoch_timing* out);
/* The same epochs as wlg_engine_run_epochs (CUDA-graph replays), with one CUDA event before
 * and one after on the engine's stream: total_ms is the device time of the whole product
 * path; walk_ms and exchange_ms are 0.  No counterpart in the reference. */
wlg_status wlg_engine_time_run(wlg_engine* engine, uint64_t epochs, wlg_epoch_timing* out);
/* Multi-walker run checkpoint (an extension: the reference checkpoints single-walker runs
 * only, src/parallel.cpp:354).  save writes every walker's full state (configuration,
 * estimators, counters, RNG), the epoch and exchange counters and the mixed-precision
 * recompute schedule, atomically (a temporary file renamed over `path`); load restores them
 * into an engine created with the same system, grid, windows, walkers, precision and
 * options, after which the run continues bit for bit as if it had not stopped.  With
 * checkpoint_path set and more than one walker, the engine restores from that file at
 * creation when it exists and writes it every checkpoint_interval_attempts. */
wlg_status wlg_engine_save_run(wlg_engine* engine, const char* path);
wlg_status wlg_engine_load_run(wlg_engine* engine, const char* path);

/* Result of the launch-shape autotuner. */
typedef struct wlg_autotune_report {
    int32_t walkers_per_block;   /* chosen walkers per CTA of the generic (CSR) sweep          */
    int32_t epochs_per_graph;    /* chosen epochs per CUDA-graph replay                        */
    double ms_per_epoch;         /* device time per epoch of the chosen shape                  */
    uint64_t trials;             /* candidate shapes timed                                     */
    int32_t staging_ring;        /* chosen staging depth of the split sweep (0: not used)      */
    int32_t pad;
} wlg_autotune_report;

/* Launch-shape autotuner: times candidate shapes (walkers per CTA 1-8 for the generic sweep,
 * epochs per graph 4-64, the split sweep's staging depth of 16 or 32 draws with their J rows
 * where both fit in shared memory) on trial_epochs real epochs each through the product path
 * and keeps the fastest.  The shape never changes results, so the trial epochs count as epochs
 * of the run.  The exchange interval, which changes trajectories, is not tuned.  No
 * counterpart in the reference. */
wlg_status wlg_engine_autotune(wlg_engine* engine, uint64_t trial_epochs, wlg_autotune_report* out);
/* Launch shape: walkers per CTA of the sweep kernel (1-8) and epochs per CUDA-graph
 * replay (>= 1); 0 leaves a value unchanged.  No counterpart in the reference. */
wlg_status wlg_engine_set_launch(wlg_engine* engine, int32_t walkers_per_block,
                                 int32_t epochs_per_graph);
/* The split sweep's staging ring (dense systems up to 1024 sites without pilot statistics or
 * the Nalivaiko mask): entries = 16 or 32 draws, each with its site's J row copied into shared
 * memory ahead of the walker; 0 restores 16.  WLG_ERR_INVALID_ARGUMENT when the engine's sweep
 * has no such ring or it does not fit.  Results do not depend on it.  No counterpart in the
 * reference. */
wlg_status wlg_engine_set_staging_ring(wlg_engine* engine, int32_t entries);
/* Single-window runs of small dense systems (one window, FP64 couplings, at most 32 sites
 * and 4 walkers, no pilot statistics or Nalivaiko mask) run many epochs per launch in one
 * CTA; this is the default for such engines.  enabled = 0 selects the per-epoch kernels
 * instead (same results); for other engines the call changes nothing.  No counterpart in
 * the reference. */
wlg_status wlg_engine_set_window_sweep(wlg_engine* engine, int32_t enabled);
/* Failure injection, for tests of the bounded device waits (no counterpart in the reference):
 * from the next epoch on, the draw-producer warps of the split sweep (dense systems up to 1024
 * sites) and of the single-window sweep publish no draws, so every walker's wait for its first
 * draws runs to its limit, the walker records WLG_ERR_TIMEOUT without writing its state back,
 * and the run call returns WLG_ERR_TIMEOUT.  Nothing faults and the device stays usable; the
 * engine itself is finished and should be destroyed.  Other sweeps are not affected. */
wlg_status wlg_engine_inject_wait_timeout(wlg_engine* engine);
/* 1 when the engine runs its epochs with the single-window kernel, else 0. */
int32_t wlg_engine_window_sweep(const wlg_engine* engine);
/* The drift report of a mixed-precision run (all zero for FP64 couplings).  No counterpart
 * in the reference. */
wlg_status wlg_engine_precision_report(wlg_engine* engine, wlg_precision_report* out);
/* Warm start before the first attempt: every walker's window slice of log g is set from
 * log_g (grid-bins entries, whole grid; finite inside every window) and its refinement
 * factor ln f to `factor` (> 0; frozen at once if <= final_factor).  No counterpart in the
 * reference, whose walkers start from log g = 0 and ln f = 1; the learned warm start
 * (replica_exchange_wang_landau_b200/warmstart.py) supplies the estimate. */
wlg_status wlg_engine_warm_start(wlg_engine* engine, const double* log_g, double factor);
/* The same warm start, continuing the 1/t schedule instead of restarting it.  Under the
 * reference's rule (begin_next_iteration, src/wang_landau.cpp:389-409) the first covered check
 * after a warm start at a small ln f switches to 1/t with f = active / attempted, far above the
 * start's factor early in a run, which discards the warm start.  Here that check halves ln f as
 * usual and then enters the 1/t stage at once from the factor reached, counting
 * round(active / factor) - attempted attempts as already made: from then on
 * f = active / (attempted + offset) (update_inverse_time_factor, src/wang_landau.cpp:309-315,
 * with the offset added): f starts from the factor reached and falls as 1/t, rising, as under
 * the reference's rule, only when the walker finds a new bin.  An extension with no
 * counterpart in the reference. */
wlg_status wlg_engine_warm_start_continue(wlg_engine* engine, const double* log_g, double factor);
uint64_t wlg_engine_walkers(const wlg_engine* engine);
uint64_t wlg_engine_bins(const wlg_engine* engine);
uint64_t wlg_engine_spins(const wlg_engine* engine);
/* Window w as (begin, end) bins. */
wlg_status wlg_engine_window(const wlg_engine* engine, uint64_t w, uint64_t* begin,
                             uint64_t* end);
/* summarize_walkers for window w (src/parallel.cpp:23-62, 170-179); arrays hold bins
 * entries.  allow_empty mirrors allow_empty_intersection. */
wlg_status wlg_engine_fragment(wlg_engine* engine, uint64_t w, int32_t allow_empty,
                               double* log_g, uint64_t* histogram, double* standard_error,
                               uint8_t* valid);
/* Every window's fragment at once (one kernel launch and one copy per array): arrays hold
 * windows x bins entries, window-major, each window's as wlg_engine_fragment gives it; the
 * first window without a common active bin fails the call unless allow_empty. */
wlg_status wlg_engine_fragments(wlg_engine* engine, int32_t allow_empty, double* log_g,
                                uint64_t* histogram, double* standard_error, uint8_t* valid);
/* summarize_sampling_impl (src/parallel.cpp:64-78). */
wlg_status wlg_engine_sampling_statistics(wlg_engine* engine, uint64_t w,
                                          double* squared_energy_displacement,
                                          uint64_t* displacement_samples,
                                          uint64_t* round_trips, uint64_t* walkers);
/* RewlResult::walker_statistics (src/parallel.cpp:541-553); capacity >= walkers. */
wlg_status wlg_engine_walker_statistics(wlg_engine* engine, wlg_walker_statistics* out,
                                        uint64_t capacity);
/* RewlResult::representatives (src/parallel.cpp:554-557): non-empty bank entries in
 * walker order; energies[capacity], spins[capacity x n]. */
wlg_status wlg_engine_representatives(wlg_engine* engine, double* energies, int8_t* spins,
                                      uint64_t capacity, uint64_t* count);

/* ---- single-walker operations (include/wl/wang_landau.hpp:98-138) -------------- */

/* WangLandauWalker::run_attempts (src/wang_landau.cpp:286-288): count attempts on walker
 * index `walker` only, without checks or exchange. */
wlg_status wlg_walker_run_attempts(wlg_engine* engine, uint64_t walker, uint64_t count);
/* snapshot / restore (src/wang_landau.cpp:415-466). */
wlg_status wlg_walker_snapshot(wlg_engine* engine, uint64_t walker, wlg_snapshot* out);
wlg_status wlg_walker_restore(wlg_engine* engine, uint64_t walker, const wlg_snapshot* in);
/* histogram_statistics / flat / covered / ready_for_iteration / begin_next_iteration
 * (src/wang_landau.cpp:344-409). */
wlg_status wlg_walker_histogram_statistics(wlg_engine* engine, uint64_t walker,
                                           wlg_histogram_statistics* out);
wlg_status wlg_walker_flags(wlg_engine* engine, uint64_t walker, int32_t* flat,
                            int32_t* covered, int32_t* ready);
wlg_status wlg_walker_begin_next_iteration(wlg_engine* engine, uint64_t walker);
/* exchange_log_probability / swap_configuration (src/wang_landau.cpp:483-508). */
wlg_status wlg_walker_exchange_log_probability(wlg_engine* engine, uint64_t left,
                                               uint64_t right, double* log_probability);
wlg_status wlg_walker_swap(wlg_engine* engine, uint64_t left, uint64_t right);

/* ---- stitching and output (wl::stitch_dos, src/analysis.cpp:45-130; write_dos_csv and
 * write_fragment_csv, src/io.cpp:398-421) ----------------------------------------------- */
/* One window's fragment: whole-grid arrays (grid-bins entries each), window [begin, end). */
typedef struct wlg_fragment_view {
    uint64_t window_begin, window_end;
    const double* log_g;
    const uint64_t* histogram;
    const double* standard_error;
    const uint8_t* valid;
} wlg_fragment_view;
/* Quality of one join (an addition: the reference reports only the join bins): over the
 * overlap of the two fragments, the number of common valid bins, the RMSE and the maximum
 * absolute difference of the aligned curves, and the slope mismatch at the join (NaN when
 * the slope criterion found no bin and the overlap midpoint was used). */
typedef struct wlg_join_quality {
    uint64_t join_bin;
    uint64_t common_bins;
    double rmse;
    double max_abs_difference;
    double slope_difference;
} wlg_join_quality;
/* Stitches `count` fragments (any order) into whole-grid outputs; joins gets count-1 entries
 * (may be NULL).  complete_range normalises sum g = 2^spin_count, else the peak is 0. */
wlg_status wlg_stitch_dos(double emin, double emax, double width, const wlg_fragment_view* fragments,
                          uint64_t count, int32_t complete_range, uint64_t spin_count, double* log_g,
                          uint64_t* histogram, double* standard_error, uint8_t* valid, wlg_join_quality* joins,
                          int32_t* fully_normalized);
/* The engine's stitched density of states: stitch_dos (src/analysis.cpp:45-130) of every
 * window's fragment, computed on the device from the fragments summarize leaves there, bit
 * for bit the curve wlg_stitch_dos gives (and the reference's stitch_dos) for the same
 * fragments.  Arrays hold grid-bins entries; joins holds windows - 1 entries (or NULL);
 * complete_range normalises sum g = 2^N (the one exp / log sum of that step runs on the host,
 * with the C library the reference uses), else the peak is 0.  The reference's errors, with
 * its messages: a window whose walkers share no active bin, adjacent fragments without a
 * common valid bin, complete_range with an invalid bin, no valid bin at all.  No counterpart
 * in the reference, which stitches on the host after run_rewl returns (apps/wl_run.cpp:180). */
wlg_status wlg_engine_stitch(wlg_engine* engine, int32_t complete_range, double* log_g, uint64_t* histogram,
                             double* standard_error, uint8_t* valid, wlg_join_quality* joins,
                             int32_t* fully_normalized);
/* The reference's <prefix>_dos.csv, byte for byte. */
wlg_status wlg_write_dos_csv(const char* path, double emin, double width, uint64_t bins, const double* log_g,
                             const uint64_t* histogram, const double* standard_error, const uint8_t* valid);
/* The reference's <prefix>_window_<w>.csv of one fragment (bins [begin, end)). */
wlg_status wlg_write_fragment_csv(const char* path, double emin, double width, uint64_t window_id,
                                  uint64_t window_begin, uint64_t window_end, const double* log_g,
                                  const uint64_t* histogram, const double* standard_error, const uint8_t* valid);
/* The reference's <prefix>_workers_stat.csv (write_workers_stat_csv, src/io.cpp:430-451), byte
 * for byte: one row per walker statistic, the MCS columns divided by spin_count (0 is
 * WLG_ERR_INVALID_ARGUMENT, "Cannot write MCS statistics for zero spins"). */
wlg_status wlg_write_workers_stat_csv(const char* path, const wlg_walker_statistics* statistics, uint64_t count,
                                      uint64_t spin_count);

/* ---- the adaptive-window pilot (apps/wl_run.cpp:104-169; src/analysis.cpp:183-420) ------ */
/* wl::AdaptiveWindowParameters (include/wl/analysis.hpp:28-38). */
typedef struct wlg_adaptive_parameters {
    uint64_t iterations;                /* pilot rounds (2)                                   */
    double pilot_mcs;                   /* MCS per pilot round (10000)                        */
    double smoothing_width;             /* energy units; 0 = automatic                        */
    double minimum_width;               /* energy units; 0 = a quarter of the mean core width */
    double diffusivity_floor_fraction;  /* 0.05                                               */
    double curvature_weight;            /* 0.25                                               */
    double round_trip_target;           /* 2                                                  */
    double maximum_round_trip_penalty;  /* 3                                                  */
} wlg_adaptive_parameters;
/* One window's pilot sampling statistics (wl::WindowSamplingStatistics), whole-grid arrays. */
typedef struct wlg_sampling_view {
    uint64_t window_begin, window_end;
    const double* squared_energy_displacement;
    const uint64_t* displacement_samples;
    uint64_t round_trips;
    uint64_t walkers;
} wlg_sampling_view;
/* adapt_energy_windows (src/analysis.cpp:183-339): windows_out gets 2*count (begin, end). */
wlg_status wlg_adapt_energy_windows(double emin, double emax, double width, const wlg_fragment_view* fragments,
                                    const wlg_sampling_view* sampling, uint64_t count, double overlap,
                                    const wlg_adaptive_parameters* parameters, uint64_t* windows_out);
/* select_adaptive_initial_configurations (src/analysis.cpp:341-420), one process: seeds for
 * count*walkers_per_window walkers (spins_out row-major, present_out 0 where none). */
wlg_status wlg_select_initial_configurations(double emin, double emax, double width, const uint64_t* windows,
                                             uint64_t count, const double* representative_energy,
                                             const int8_t* representative_spins, const uint8_t* representative_present,
                                             uint64_t representatives, uint64_t spins, uint64_t walkers_per_window,
                                             int8_t* spins_out, uint8_t* present_out, uint64_t* missing,
                                             uint64_t* external);

/* ---- batches of engines (no counterpart in the reference, which runs one instance) -----
 * Engines created on the same device (different systems, sizes, windows or precisions)
 * advanced together: one CUDA graph whose child graphs are the engines' captured epoch
 * graphs, so a single launch runs every engine's next epochs side by side on the GPU.  An
 * engine that has terminated keeps running no-op epochs.  Creating a batch runs one epoch
 * of every engine whose epoch graph did not exist yet.  The engines must outlive the batch
 * and must not be used elsewhere while wlg_batch_run_epochs runs. */
typedef struct wlg_batch wlg_batch;
wlg_status wlg_batch_create(wlg_engine* const* engines, uint64_t count, wlg_batch** out);
/* Launches until every engine has terminated or about max_epochs epochs have run (each launch
 * advances every engine by its epochs per graph); *launches = graph launches made. */
wlg_status wlg_batch_run_epochs(wlg_batch* batch, uint64_t max_epochs, uint64_t* launches, int32_t* all_done);
void wlg_batch_destroy(wlg_batch* batch);

/* ---- the warm-start network (no counterpart in the reference) --------------------------
 * A small multilayer perceptron trained on DOS curves that plain runs produce: inputs are
 * per-bin features of a system (replica_exchange_wang_landau_b200/warmstart.py), the output
 * is log g per spin.  Fully connected layers, tanh on hidden layers, identity output, mean
 * squared error, full-batch Adam; forward, backward and the optimiser run as hand-written
 * CUDA kernels.  Parameters are FP32 in one array: for each layer l, W_l (dims[l+1] x
 * dims[l], row-major) then b_l (dims[l+1]).  Host buffers in and out. */
typedef struct wlg_mlp wlg_mlp;
/* layers = number of weight layers (1-8); dims has layers+1 widths (1-4096), dims[layers]
 * = 1.  Glorot-uniform weights from a splitmix64 stream of `seed`, zero biases. */
wlg_status wlg_mlp_create(int32_t layers, const int32_t* dims, uint64_t seed, wlg_mlp** out);
void wlg_mlp_destroy(wlg_mlp* mlp);
uint64_t wlg_mlp_parameter_count(const wlg_mlp* mlp);
wlg_status wlg_mlp_get_parameters(wlg_mlp* mlp, float* out);
/* Also resets the optimiser state. */
wlg_status wlg_mlp_set_parameters(wlg_mlp* mlp, const float* in);
/* y[batch] = network(x[batch x dims[0]]). */
wlg_status wlg_mlp_forward(wlg_mlp* mlp, const float* x, uint64_t batch, float* y);
/* Mean squared error against t[batch] and its gradient with respect to every parameter,
 * at the current parameters (no update). */
wlg_status wlg_mlp_gradients(wlg_mlp* mlp, const float* x, const float* t, uint64_t batch, float* grads,
                             double* loss);
/* `steps` full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8); *loss = the error after
 * the last step. */
wlg_status wlg_mlp_train(wlg_mlp* mlp, const float* x, const float* t, uint64_t batch, uint64_t steps,
                         double learning_rate, double* loss);

#ifdef __cplusplus
}
#endif

#endif /* WLG_H */
