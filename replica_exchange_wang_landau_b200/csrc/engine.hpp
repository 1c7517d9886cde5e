// engine.hpp — host side of the REWL engine: device buffers, the Engine class that owns a
// run (the replacement of run_rewl, src/parallel.cpp:276-747) and the kernel launchers.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wlg.h"
#include "common.cuh"

namespace wlg {

// An error carrying a wlg_status; the C-ABI layer turns it into a return code + message.
struct WlgError : std::runtime_error {
    wlg_status status;
    WlgError(wlg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw WlgError(WLG_ERR_DEVICE, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// The stream on which the current device's buffers are allocated and freed, from a memory
// pool of the library's own (not the device's default pool).  Created once per device and
// kept; the pool keeps freed memory (release threshold = unlimited) so that creating and
// destroying engines costs no driver-level allocation after the first one.  (cudaMalloc /
// cudaFree took up to hundreds of ms per engine destruction.)
cudaStream_t pool_stream();
// `bytes` from that pool, complete when the call returns.
void* pool_allocate(size_t bytes);

// Owning device allocation, stream-ordered on pool_stream().  The allocation is complete
// before allocate() returns, so any stream may use it.  The owner must have finished every
// use of the buffer when it is released (the engine and the helpers synchronise their stream
// first); while an exception unwinds, release() synchronises the device before freeing, so a
// kernel left in flight by the error cannot write into reused memory.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t b) { allocate(b); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes), stream(o.stream) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    ~DeviceBuffer() { release(); }
    void allocate(size_t b) {
        release();
        if (b == 0) b = 16;
        ptr = pool_allocate(b);
        stream = pool_stream();
        bytes = b;
    }
    void release() {
        if (ptr) {
            if (std::uncaught_exceptions() > 0) cudaDeviceSynchronize();
            cudaFreeAsync(ptr, stream);
        }
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T* get() const { return static_cast<T*>(ptr); }
};

// A system resident on the device: geometry plus the couplings built from it.
struct DeviceSystem {
    uint64_t n = 0;
    uint64_t ld = 0;  // padded stride, multiple of 16
    double box[3] = {0, 0, 0};
    int32_t periodic = 0;
    double scale = 1.0;
    double cutoff = 0.0;
    bool csr = false;
    uint64_t nnz = 0;
    DeviceBuffer pos, axes;
    DeviceBuffer J64, J32, J16, Jscale;
    DeviceBuffer csr_ptr, csr_col, csr_val64, csr_val32;
    DeviceBuffer ell_col, ell_val64, ell_val32;  // ELLPACK rows for the CSR sweep
    int32_t ell_width = 0;                       // entries per row (0: not built)
    // cell grid of the CSR build: sites sorted by cell, cells at least the cutoff wide
    DeviceBuffer cell_start, cell_sites, site_cell;
    int32_t cells[3] = {1, 1, 1};
    int32_t cell_wrap[3] = {0, 0, 0};
};

// Host-side validation and helpers (host.cpp).
void validate_system(const wlg_system& s);
void validate_grid(double emin, double emax, double width);
uint64_t grid_bins(double emin, double emax, double width);
std::vector<uint64_t> partition_windows(uint64_t bins, uint64_t count, double overlap);
void upload_system(const wlg_system& s, DeviceSystem& d, cudaStream_t stream);
// Prebuilt couplings: validated (symmetric, zero diagonal, finite; CSR rows sorted by column)
// and uploaded in the layouts build_couplings produces.
void validate_couplings(const wlg_couplings& j);
void upload_couplings(const wlg_couplings& j, DeviceSystem& d, int precision, cudaStream_t stream);
void upload_cell_grid(const wlg_system& s, DeviceSystem& d, cudaStream_t stream);
void save_checkpoint_file(const std::string& path, const wlg_snapshot& s, uint64_t n, uint64_t bins);
bool load_checkpoint_file(const std::string& path, std::vector<int8_t>& spins, std::vector<double>& fields,
                          std::vector<double>& log_g, std::vector<uint64_t>& hist, std::vector<uint8_t>& active,
                          wlg_snapshot& scalars, std::string& error);

// adaptive.cpp
std::vector<uint64_t> adapt_energy_windows(double emin, double emax, double width, const wlg_fragment_view* fragments,
                                           const wlg_sampling_view* sampling, uint64_t count, double overlap,
                                           const wlg_adaptive_parameters& p);
void select_initial_configurations(double emin, double emax, double width, const uint64_t* windows, uint64_t count,
                                   const double* rep_energy, const int8_t* rep_spins, const uint8_t* rep_present,
                                   uint64_t reps, uint64_t n, uint64_t walkers_per_window, int8_t* spins_out,
                                   uint8_t* present_out, uint64_t* missing, uint64_t* external);

// stitch.cpp
void stitch_dos(double emin, double emax, double width, const wlg_fragment_view* fragments, uint64_t count,
                bool complete_range, uint64_t spins, double* log_g, uint64_t* histogram, double* standard_error,
                uint8_t* valid, wlg_join_quality* joins, int32_t* fully_normalized);
void write_dos_csv(const char* path, double emin, double width, uint64_t bins, const double* log_g,
                   const uint64_t* histogram, const double* standard_error, const uint8_t* valid);
void write_fragment_csv(const char* path, double emin, double width, uint64_t window_id, uint64_t begin,
                        uint64_t end, const double* log_g, const uint64_t* histogram, const double* standard_error,
                        const uint8_t* valid);
void write_workers_stat_csv(const char* path, const wlg_walker_statistics* stats, uint64_t count,
                            uint64_t spin_count);

// physics.cu
void build_couplings(DeviceSystem& d, int precision, cudaStream_t stream);
// noalloc.cu: local fields with every intermediate in a static device array.
void local_fields_noalloc(const wlg_system& s, const int8_t* spins, uint64_t count, double* fields,
                          double* energies);
// dense_build_kernel on caller-provided device buffers (J is ld x ld and must be zeroed).
void launch_dense_build(const double* pos, const double* axes, const double* box, int periodic, double scale, int n,
                        int ld, double* J, int* err, cudaStream_t stream);
void compute_fields(const EngineView& v, const int8_t* spins, int64_t spin_stride, double* fields,
                    int64_t field_stride, double* energies, int count, cudaStream_t stream);

// Per-walker result of the target-Metropolis initialisation (the numbers the reference's
// failure message prints, src/wang_landau.cpp:221-241).
struct InitReport {
    int32_t status;  // 0 ok, 1 did not reach the target band
    int32_t pad;
    double target;
    double half_width;
    double minimum_reached;
    double maximum_reached;
    double closest;
    double closest_distance;
    double highest_temperature;
    uint64_t increases;
    uint64_t restarts;
    uint64_t stall;
};

struct WalkArgs {
    int32_t first;          // first walker of the launch
    int32_t count;          // walkers in the launch
    uint64_t fixed_batch;   // > 0: exactly this many attempts, no check (run_attempts)
    int32_t epoch_mode;     // 1: run_rewl batch + check + termination counters
    int32_t smem_per_walker;
};

struct InitArgs {
    int32_t smem_per_walker;
    int32_t pad;
    const int8_t* initial_spins;   // walkers x ld or null
    const uint8_t* present;        // per walker
    InitReport* reports;
    uint64_t init_max_attempts;
    double target_fraction;
    double temperature_fraction;
    uint64_t stall_per_spin;
    double temperature_multiplier;
    double max_temperature_fraction;
};

// walker.cu
size_t walker_smem_bytes(const EngineView& v, bool smem_fields, bool features);
bool fields_fit_in_smem(const EngineView& v, bool features);
void launch_init(const EngineView& v, const InitArgs& a, int walkers_per_block, cudaStream_t stream);
void launch_walk(const EngineView& v, const WalkArgs& a, int walkers_per_block, cudaStream_t stream);
// sweep.cu: the dense sweep; false when the walker does not fit the shared-memory ring.
bool launch_sweep_dense(const EngineView& v, const WalkArgs& a, cudaStream_t stream);
// The split sweep's possible staging depths for this engine (log2 of the draw / J-row ring);
// empty when the split sweep does not serve it.
std::vector<int> split_ring_logs(const EngineView& v);
bool launch_sweep_csr(const EngineView& v, const WalkArgs& a, int walkers_per_block, cudaStream_t stream);
// sweep_window.cu: whole epochs of a single-window run of a dense FP64 system of at most 32
// sites and 4 walkers, without pilot statistics or the Nalivaiko mask, in one launch
bool window_sweep_fits(const EngineView& v);
void launch_sweep_window(const EngineView& v, uint32_t epochs, cudaStream_t stream);
void launch_ell_fill(int n, int width, const int32_t* ptr, const int32_t* col, const double* val64,
                     const float* val32, int32_t* ell_col, double* ell_val64, float* ell_val32, cudaStream_t stream);
void launch_exchange(const EngineView& v, cudaStream_t stream);
// precision.cu: drift measurement and resync after an FP64 recompute of all fields.
void launch_resync(const EngineView& v, const double* rfields, const double* renergy, PrecisionReport* report,
                   cudaStream_t stream);
void launch_flush_pending(const EngineView& v, cudaStream_t stream);
// summarize_impl for windows [window, window + windows): outputs window-major, bins each
void launch_summarize(const EngineView& v, int window, int windows, int allow_empty, double* log_g, uint64_t* hist,
                      double* sem, uint8_t* valid, int* status, cudaStream_t stream);
// stitch.cu: stitch_dos on the fragments summarize_kernel left on the device.  Status codes:
constexpr int kStitchNoCommonBin = 1;          // "Walkers in an energy window have no common active bin"
constexpr int kStitchNoOverlap = 2;            // "DOS fragments must overlap and match the global grid"
constexpr int kStitchNoCommonOverlapBin = 3;   // "Adjacent DOS fragments have no common valid overlap bin"
constexpr int kStitchIncomplete = 4;           // "Complete-range normalization requires every DOS bin to be valid"
constexpr int kStitchNoValidBins = 5;          // "Stitched DOS has no valid bins"
void launch_stitch(int windows, int bins, const int32_t* wbeg, const int32_t* wend, const double* flg,
                   const uint64_t* fh, const double* fse, const uint8_t* fv, const int* summarize_status,
                   double width, int complete_range, double* lg, uint64_t* h, double* se, uint8_t* ok,
                   wlg_join_quality* joins, int* status, cudaStream_t stream);
void launch_sampling(const EngineView& v, int window, double* sq, uint64_t* samples, uint64_t* trips,
                     cudaStream_t stream);
void launch_walker_statistics(const EngineView& v, wlg_walker_statistics* out, cudaStream_t stream);
void launch_histogram_statistics(const EngineView& v, int walker, wlg_histogram_statistics* out, int* flags,
                                 cudaStream_t stream);
void launch_begin_next_iteration(const EngineView& v, int walker, int* status, cudaStream_t stream);
void launch_exchange_pair(const EngineView& v, int left, int right, int do_swap, double* logp, int* status,
                          cudaStream_t stream);

// mlp.cu: the warm-start network (forward, backward and Adam on the device).
class Mlp;
Mlp* mlp_create(int layers, const int32_t* dims, uint64_t seed);
void mlp_destroy(Mlp* m);
size_t mlp_count(const Mlp* m);
void mlp_get(Mlp* m, float* out);
void mlp_set(Mlp* m, const float* in);
void mlp_forward(Mlp* m, const float* x, uint64_t batch, float* y);
double mlp_gradients(Mlp* m, const float* x, const float* t, uint64_t batch, float* g);
double mlp_train(Mlp* m, const float* x, const float* t, uint64_t batch, uint64_t steps, double lr);

class Engine;

// Several engines on one device advanced together: one CUDA graph whose child graphs are the
// engines' captured epoch graphs, so one launch runs every instance's epochs side by side.
class Batch {
  public:
    explicit Batch(const std::vector<Engine*>& engines);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    void run_epochs(uint64_t max_epochs, uint64_t* launches, int32_t* all_done);

  private:
    std::vector<Engine*> engines_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaStream_t stream_ = nullptr;
    uint64_t epochs_per_launch_ = 1;
};

// The engine: one REWL run on the current device.
class Engine {
  public:
    Engine(const wlg_system& system, const wlg_run_config& config);
    // From prebuilt couplings (no geometry): the J a Couplings object exports.
    Engine(const wlg_couplings& couplings, const wlg_run_config& config);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    void run(wlg_run_totals* totals);
    void run_epochs(uint64_t max_epochs, uint64_t* epochs_run, int32_t* done);
    void totals(wlg_run_totals* out);
    void time_epochs(uint64_t epochs, wlg_epoch_timing* out);
    void time_run(uint64_t epochs, wlg_epoch_timing* out);
    void autotune(uint64_t trial_epochs, wlg_autotune_report* out);
    void set_launch(int walkers_per_block, int epochs_per_graph);
    // the split sweep's staging ring (draws with their J rows): 16 or 32 entries, 0 = 16
    void set_staging_ring(int entries);
    int staging_ring() const;
    // Failure injection for tests: from the next epoch on, the draw producers of the split and
    // single-window sweeps publish nothing, so every walker's bounded wait runs out.
    void inject_wait_timeout();
    uint64_t walkers() const { return walkers_; }
    uint64_t bins() const { return bins_; }
    uint64_t spins() const { return sys_.n; }
    void window(uint64_t w, uint64_t* begin, uint64_t* end) const;
    void fragment(uint64_t w, int allow_empty, double* log_g, uint64_t* hist, double* sem, uint8_t* valid);
    // every window's fragment in one launch and one copy (arrays windows x bins, window-major)
    void fragments(int allow_empty, double* log_g, uint64_t* hist, double* sem, uint8_t* valid);
    // stitch_dos of every window's fragment on the device (whole-grid outputs, bins entries;
    // joins: windows - 1 entries or NULL)
    void stitch(int complete_range, double* log_g, uint64_t* hist, double* sem, uint8_t* valid,
                wlg_join_quality* joins, int32_t* fully_normalized);
    void sampling(uint64_t w, double* sq, uint64_t* samples, uint64_t* round_trips, uint64_t* walkers);
    void walker_statistics(wlg_walker_statistics* out, uint64_t capacity);
    void representatives(double* energies, int8_t* spins, uint64_t capacity, uint64_t* count);

    void run_attempts(uint64_t walker, uint64_t count);
    void snapshot(uint64_t walker, wlg_snapshot* out);
    void restore(uint64_t walker, const wlg_snapshot& in);
    void histogram_statistics(uint64_t walker, wlg_histogram_statistics* out, int32_t* flags);
    void begin_next_iteration(uint64_t walker);
    double exchange_log_probability(uint64_t left, uint64_t right);
    void swap(uint64_t left, uint64_t right);
    void precision_report(wlg_precision_report* out);
    // continue_schedule: the first covered check enters the 1/t stage at the factor reached and
    // counts round(active / factor) attempts as made (f = active / (attempted + offset)), so the
    // factor starts where the warm start left it; false keeps the reference's rule.
    void warm_start(const double* log_g, double factor, bool continue_schedule = false);
    // every walker's state, the control block and the recompute schedule (multi-walker
    // checkpoint; the reference checkpoints single-walker runs only)
    void save_run(const std::string& path);
    void load_run(const std::string& path);
    // batch support: the captured epoch graph (built on first use, after one direct epoch that
    // primes the kernels) and the host work after epochs that a batch launch ran
    cudaGraph_t epoch_graph();
    void after_external_epochs();
    bool is_done() const { return done_; }
    uint64_t epoch_count() const { return epochs_; }

    // Launch shape (chosen by the autotuner or set explicitly).
    int walkers_per_block = 1;
    int epochs_per_graph = 32;
    // Single-window runs of small dense systems: whole epochs per launch (sweep_window.cu).
    // Eligibility is fixed at creation; set_window_sweep(false) selects the per-epoch kernels.
    bool window_sweep_eligible() const { return window_sweep_eligible_; }
    bool window_sweep() const { return window_sweep_; }
    void set_window_sweep(bool on) { window_sweep_ = on && window_sweep_eligible_; }
    int device = 0;  // CUDA device the engine lives on

  private:
    void configure(const wlg_run_config& c);
    void check_backend(bool csr) const;
    void initialise_walkers(const wlg_run_config& c);
    void check_device_error();
    void launch_epochs(uint64_t count);
    void build_graph();
    void maybe_checkpoint();
    void recompute_fields();
    void launch_recompute();
    void launch_epoch(const WalkArgs& a);
    void after_epochs();
    void finish();
    void print_progress(bool final_line);
    std::vector<WalkerState> download_states();

    bool window_sweep_eligible_ = false;
    bool window_sweep_ = false;
    wlg_run_config cfg_{};
    DeviceParams p_{};
    DeviceSystem sys_;
    Grid grid_{};
    uint64_t bins_ = 0, windows_ = 0, wpw_ = 0, walkers_ = 0;
    std::vector<uint64_t> win_;  // 2 * windows
    bool features_ = false;
    bool smem_fields_ = true;
    int precision_ = WLG_PRECISION_FP64;
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    int graph_epochs_ = 0;

    DeviceBuffer d_win_begin_, d_win_end_, d_ws_, d_log_g_, d_hist_, d_active_, d_refine_, d_sqdisp_,
        d_dsamples_, d_spins_, d_fields_, d_rep_energy_, d_rep_dist_, d_rep_target_, d_rep_present_,
        d_rep_spins_, d_ctl_, d_scratch_, d_frag_, d_stitch_;
    // mixed precision: FP64 recompute every recompute_epochs_ epochs (0 = never)
    DeviceBuffer d_rfields_, d_renergy_, d_prec_;
    uint64_t recompute_epochs_ = 0, next_recompute_ = 0;
    EngineView view_{};

    std::string checkpoint_path_;
    bool checkpointing_ = false;
    uint64_t last_checkpoint_ = 0;
    bool done_ = false;
    bool finished_ = false;
    bool checkpointing_all_ = false;  // more than one walker: the multi-walker format
    uint64_t system_hash_ = 0;
    uint64_t epochs_ = 0;
    double next_progress_ = 0.0;
    size_t progress_width_ = 0;
};

}  // namespace wlg
