// engine.cpp — the REWL run on one GPU: the replacement of run_rewl (src/parallel.cpp:276-747).
//
// Set-up mirrors run_rewl's: validate the configuration, partition the windows, construct
// walkers (init_kernel), restore a single-walker checkpoint.  The epoch loop is a sequence
// of [walk_kernel -> exchange_kernel] pairs captured once in a CUDA graph and replayed; the
// device keeps the epoch counter and the termination flag, so a replay after termination is
// a sequence of no-op launches and the host only reads the control block between replays.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <mutex>
#include <sstream>

#include "engine.hpp"

namespace wlg {

namespace {

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The WlParameters checks of the WangLandauWalker constructor (src/wang_landau.cpp:74-90).
bool parameters_valid(const wlg_wl_parameters& p) {
    return (p.flatness > 0.0 && p.flatness <= 1.0) && (p.final_factor > 0.0) && p.check_interval_attempts != 0 &&
           p.initialization_max_attempts != 0 &&
           (p.initialization_target_fraction > 0.0 && p.initialization_target_fraction <= 1.0) &&
           std::isfinite(p.initialization_temperature_fraction) && (p.initialization_temperature_fraction > 0.0) &&
           p.initialization_stall_attempts_per_spin != 0 && std::isfinite(p.initialization_temperature_multiplier) &&
           (p.initialization_temperature_multiplier > 1.0) &&
           std::isfinite(p.initialization_max_temperature_fraction) &&
           !(p.initialization_max_temperature_fraction < p.initialization_temperature_fraction) &&
           std::isfinite(p.round_trip_margin_fraction) && !(p.round_trip_margin_fraction < 0.0) &&
           !(p.round_trip_margin_fraction >= 0.5);
}

// The device check, once per device (cudaGetDeviceProperties alone took 8-60 ms per call).
void require_device() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw WlgError(WLG_ERR_DEVICE, "No CUDA device is available; this engine runs on an sm_100 (B200) GPU only");
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    static std::atomic<uint64_t> checked{0};
    if (device < 64 && (checked.load() >> device & 1)) return;
    int major = 0;
    check_cuda(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "cudaDeviceGetAttribute");
    if (major != 10) {
        cudaDeviceProp prop{};
        check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        throw WlgError(WLG_ERR_DEVICE, std::string("This engine is built for sm_100a (B200); found ") + prop.name);
    }
    if (device < 64) checked.fetch_or(uint64_t{1} << device);
}

}  // namespace

namespace {

struct DevicePool {
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
};

// The library's own stream and memory pool on the current device, created once.  The pool
// is private: the device's default pool, which other code in the process may use through
// cudaMallocAsync, keeps its own attributes.
const DevicePool& device_pool() {
    static std::mutex mu;
    static DevicePool pools[64];
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= 64) throw WlgError(WLG_ERR_DEVICE, "device index beyond 63");
    std::lock_guard<std::mutex> lock(mu);
    DevicePool& d = pools[device];
    if (!d.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        check_cuda(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = ~0ULL;
        check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        check_cuda(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        d.pool = pool;
    }
    return d;
}

}  // namespace

cudaStream_t pool_stream() { return device_pool().stream; }

void* pool_allocate(size_t bytes) {
    const DevicePool& d = device_pool();
    void* ptr = nullptr;
    check_cuda(cudaMallocFromPoolAsync(&ptr, bytes, d.pool, d.stream), "cudaMallocFromPoolAsync");
    check_cuda(cudaStreamSynchronize(d.stream), "allocation");
    return ptr;
}

Engine::Engine(const wlg_system& system, const wlg_run_config& c) : cfg_(c) {
    configure(c);
    validate_system(system);
    check_backend(system.cutoff > 0.0);
    // fingerprint of the system, so that a run checkpoint is never restored onto another one
    {
        uint64_t h = 1469598103934665603ULL;
        auto mix = [&h](const void* p, size_t bytes) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            for (size_t k = 0; k < bytes; ++k) h = (h ^ c[k]) * 1099511628211ULL;
        };
        mix(system.positions, system.n * 24);
        mix(system.axes, system.n * 24);
        mix(system.box, sizeof system.box);
        mix(&system.periodic, sizeof system.periodic);
        mix(&system.coupling_scale, sizeof system.coupling_scale);
        mix(&system.cutoff, sizeof system.cutoff);
        system_hash_ = h;
    }
    require_device();
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    upload_system(system, sys_, stream_);
    build_couplings(sys_, precision_, stream_);
    initialise_walkers(c);
}

Engine::Engine(const wlg_couplings& couplings, const wlg_run_config& c) : cfg_(c) {
    configure(c);
    validate_couplings(couplings);
    check_backend(couplings.dense == nullptr);
    // fingerprint of the couplings (a different domain from the geometry fingerprint)
    {
        uint64_t h = 0x9e3779b97f4a7c15ULL;
        auto mix = [&h](const void* p, size_t bytes) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            for (size_t k = 0; k < bytes; ++k) h = (h ^ c[k]) * 1099511628211ULL;
        };
        const uint64_t n = couplings.n;
        mix(&n, sizeof n);
        if (couplings.dense) {
            mix(couplings.dense, n * n * 8);
        } else {
            mix(couplings.row_offsets, (n + 1) * 8);
            mix(couplings.columns, couplings.nnz * 8);
            mix(couplings.values, couplings.nnz * 8);
        }
        system_hash_ = h;
    }
    require_device();
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    upload_couplings(couplings, sys_, precision_, stream_);
    initialise_walkers(c);
}

void Engine::check_backend(bool csr) const {
    if (csr && precision_ == WLG_PRECISION_BF16)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "BF16 couplings are available for the dense backend only");
}

// The run configuration: RunConfig::validate (src/io.cpp:243-268), as run_rewl calls it, the
// grid and windows, and the parameters the kernels read.
void Engine::configure(const wlg_run_config& c) {
    if (!std::isfinite(c.progress_interval_seconds) || c.progress_interval_seconds < 0.0 || c.windows == 0 ||
        c.walkers_per_window == 0 || c.overlap < 0.0 || c.overlap >= 1.0 || c.exchange_interval_attempts == 0 ||
        c.wl.check_interval_attempts == 0 || c.checkpoint_interval_attempts == 0 ||
        !std::isfinite(c.wl.round_trip_margin_fraction) || c.wl.round_trip_margin_fraction < 0.0 ||
        c.wl.round_trip_margin_fraction >= 0.5)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid run configuration");
    validate_grid(c.emin, c.emax, c.bin_width);
    bins_ = grid_bins(c.emin, c.emax, c.bin_width);
    if (c.windows > bins_) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "More windows than energy bins");
    if (c.explicit_windows) {
        const uint64_t* e = c.explicit_windows;
        if (e[0] != 0 || e[2 * c.windows - 1] != bins_)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Explicit energy windows must match the configured range");
        for (uint64_t i = 0; i < c.windows; ++i)
            if (e[2 * i] >= e[2 * i + 1] || e[2 * i + 1] > bins_ ||
                (i != 0 && (e[2 * i] <= e[2 * (i - 1)] || e[2 * i] >= e[2 * (i - 1) + 1])))
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Explicit energy windows must be ordered and overlap");
        win_.assign(e, e + 2 * c.windows);
    } else {
        win_ = partition_windows(bins_, c.windows, c.overlap);
    }
    if (c.coupling_precision < WLG_PRECISION_FP64 || c.coupling_precision > WLG_PRECISION_BF16)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Unknown coupling precision");
    if (c.windows * c.walkers_per_window > static_cast<uint64_t>(std::numeric_limits<int32_t>::max() / 64))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Too many walkers");
    if (bins_ > static_cast<uint64_t>(std::numeric_limits<int32_t>::max() / 2))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Too many energy bins");

    windows_ = c.windows;
    wpw_ = c.walkers_per_window;
    walkers_ = windows_ * wpw_;
    precision_ = c.coupling_precision;
    grid_ = make_grid(c.emin, c.emax, c.bin_width, static_cast<int64_t>(bins_));
    features_ = c.wl.collect_window_statistics != 0 || c.wl.nalivaiko_mod != 0;

    p_.flatness = c.wl.flatness;
    p_.minimum_visits = c.wl.minimum_visits;
    p_.final_factor = c.wl.final_factor;
    p_.check_interval = std::max<uint64_t>(1, c.wl.check_interval_attempts);
    p_.force_after = c.wl.force_accept_after_attempts;
    p_.inverse_time = c.wl.inverse_time_enabled != 0;
    p_.nalivaiko = c.wl.nalivaiko_mod != 0;
    p_.collect = c.wl.collect_window_statistics != 0;
    p_.round_trip_margin = c.wl.round_trip_margin_fraction;
    p_.exchange_interval = c.exchange_interval_attempts;
    p_.max_attempts = c.max_attempts;
    p_.seed = c.seed;
    if (c.checkpoint_path && c.checkpoint_path[0]) checkpoint_path_ = c.checkpoint_path;
    cfg_.explicit_windows = nullptr;
    cfg_.initial_spins = nullptr;
    cfg_.initial_spins_present = nullptr;
    cfg_.checkpoint_path = nullptr;
}

Engine::~Engine() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
}

void Engine::initialise_walkers(const wlg_run_config& c) {
    const uint64_t n = sys_.n, ld = sys_.ld, W = walkers_, B = bins_;
    uint64_t mwb = 0;
    for (uint64_t w = 0; w < windows_; ++w) mwb = std::max(mwb, win_[2 * w + 1] - win_[2 * w]);

    std::vector<int32_t> wb(windows_), we(windows_);
    for (uint64_t w = 0; w < windows_; ++w) {
        wb[w] = static_cast<int32_t>(win_[2 * w]);
        we[w] = static_cast<int32_t>(win_[2 * w + 1]);
    }
    d_win_begin_.allocate(windows_ * sizeof(int32_t));
    d_win_end_.allocate(windows_ * sizeof(int32_t));
    check_cuda(cudaMemcpyAsync(d_win_begin_.ptr, wb.data(), windows_ * 4, cudaMemcpyHostToDevice, stream_), "copy");
    check_cuda(cudaMemcpyAsync(d_win_end_.ptr, we.data(), windows_ * 4, cudaMemcpyHostToDevice, stream_), "copy");

    auto zeroed = [&](DeviceBuffer& b, size_t bytes) {
        b.allocate(bytes);
        check_cuda(cudaMemsetAsync(b.ptr, 0, b.bytes, stream_), "memset");
    };
    zeroed(d_ws_, W * sizeof(WalkerState));
    zeroed(d_log_g_, W * B * sizeof(double));
    zeroed(d_hist_, W * B * sizeof(uint64_t));
    zeroed(d_active_, W * B);
    zeroed(d_refine_, features_ ? W * B : 16);
    zeroed(d_sqdisp_, features_ ? W * B * sizeof(double) : 16);
    zeroed(d_dsamples_, features_ ? W * B * sizeof(uint64_t) : 16);
    zeroed(d_spins_, W * ld);
    zeroed(d_fields_, W * ld * sizeof(double));
    const uint64_t R = p_.collect ? W * kRepresentatives : 1;
    zeroed(d_rep_energy_, R * sizeof(double));
    zeroed(d_rep_dist_, R * sizeof(double));
    zeroed(d_rep_target_, R * sizeof(double));
    zeroed(d_rep_present_, R);
    zeroed(d_rep_spins_, p_.collect ? R * ld : 16);
    zeroed(d_ctl_, sizeof(Control));
    zeroed(d_prec_, sizeof(PrecisionReport));
    if (precision_ != WLG_PRECISION_FP64 && c.recompute_interval_attempts != 0) {
        // the recompute runs at the first exchange boundary after every interval
        recompute_epochs_ = std::max<uint64_t>(
            1, (c.recompute_interval_attempts + c.exchange_interval_attempts - 1) / c.exchange_interval_attempts);
        next_recompute_ = recompute_epochs_;
        d_rfields_.allocate(W * ld * sizeof(double));
        d_renergy_.allocate(W * sizeof(double));
    }
    d_scratch_.allocate(std::max<size_t>(B * 32 + 256, W * sizeof(wlg_walker_statistics) + 256));

    EngineView& v = view_;
    v.n = static_cast<int32_t>(n);
    v.ld = static_cast<int32_t>(ld);
    v.site_mod = make_fastmod(n);
    v.precision = precision_;
    v.csr = sys_.csr ? 1 : 0;
    v.J64 = sys_.J64.get<double>();
    v.J32 = sys_.J32.get<float>();
    v.J16 = sys_.J16.get<__nv_bfloat16>();
    v.Jscale = sys_.Jscale.get<float>();
    v.csr_ptr = sys_.csr_ptr.get<int32_t>();
    v.csr_col = sys_.csr_col.get<int32_t>();
    v.csr_val64 = sys_.csr_val64.get<double>();
    v.csr_val32 = sys_.csr_val32.get<float>();
    v.ell_col = sys_.ell_col.get<int32_t>();
    v.ell_val64 = sys_.ell_val64.get<double>();
    v.ell_val32 = sys_.ell_val32.get<float>();
    v.ell_width = sys_.ell_width;
    v.grid = grid_;
    v.walkers = static_cast<int32_t>(W);
    v.walkers_per_window = static_cast<int32_t>(wpw_);
    v.windows = static_cast<int32_t>(windows_);
    v.max_window_bins = static_cast<int32_t>(mwb);
    v.win_begin = d_win_begin_.get<int32_t>();
    v.win_end = d_win_end_.get<int32_t>();
    v.ws = d_ws_.get<WalkerState>();
    v.log_g = d_log_g_.get<double>();
    v.hist = d_hist_.get<uint64_t>();
    v.active = d_active_.get<uint8_t>();
    v.refine = d_refine_.get<uint8_t>();
    v.sqdisp = d_sqdisp_.get<double>();
    v.dsamples = d_dsamples_.get<uint64_t>();
    v.spins = d_spins_.get<int8_t>();
    v.fields = d_fields_.get<double>();
    v.rep_energy = d_rep_energy_.get<double>();
    v.rep_dist = d_rep_dist_.get<double>();
    v.rep_target = d_rep_target_.get<double>();
    v.rep_present = d_rep_present_.get<uint8_t>();
    v.rep_spins = d_rep_spins_.get<int8_t>();
    v.p = p_;
    v.ctl = d_ctl_.get<Control>();

    v.spins_global = 0;
    smem_fields_ = !sys_.csr || fields_fit_in_smem(v, features_);
    // a large cutoff system keeps the spins of the initialisation and the generic sweep in HBM
    if (sys_.csr && !smem_fields_ && walker_smem_bytes(v, false, features_) > 200 * 1024) v.spins_global = 1;
    if (!sys_.csr && !fields_fit_in_smem(v, features_))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Dense system too large for the shared-memory walker (use a cutoff)");
    window_sweep_eligible_ = window_sweep_fits(v);
    window_sweep_ = window_sweep_eligible_;

    // Host-prepared walker headers: window, slot, representative targets (ctor lines 104-118).
    std::vector<WalkerState> states(W);
    std::vector<double> targets(R, 0.0), dist(R, std::numeric_limits<double>::infinity());
    for (uint64_t w = 0; w < W; ++w) {
        WalkerState& s = states[w];
        std::memset(&s, 0, sizeof s);
        s.window = static_cast<int32_t>(w / wpw_);
        s.slot = static_cast<int32_t>(w);
        s.factor = 1.0;
        s.cur_bin = -1;
        if (p_.collect) {
            const double lower = c.emin + static_cast<double>(win_[2 * s.window]) * c.bin_width;
            const double upper = c.emin + static_cast<double>(win_[2 * s.window + 1]) * c.bin_width;
            targets[w * kRepresentatives] = lower;
            for (int r = 1; r < kRepresentatives; ++r)
                targets[w * kRepresentatives + r] =
                    lower + (upper - lower) * (static_cast<double>(r) - 0.5) / static_cast<double>(kRepresentatives - 1);
        }
    }
    check_cuda(cudaMemcpyAsync(d_ws_.ptr, states.data(), W * sizeof(WalkerState), cudaMemcpyHostToDevice, stream_),
               "copy states");
    if (p_.collect) {
        check_cuda(cudaMemcpyAsync(d_rep_target_.ptr, targets.data(), R * 8, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaMemcpyAsync(d_rep_dist_.ptr, dist.data(), R * 8, cudaMemcpyHostToDevice, stream_), "copy");
    }

    // Per-walker construction errors that the reference raises inside the constructor
    // (src/wang_landau.cpp:70-96) are reported as that walker's initialisation failure.
    auto ctor_failure = [&](uint64_t w, const std::string& what) {
        std::ostringstream m;
        m << "Walker initialization failed: window " << w / wpw_ << ", local walker " << w % wpw_ << ": " << what;
        throw WlgError(WLG_ERR_INIT_FAILED, m.str());
    };
    if (!parameters_valid(c.wl)) ctor_failure(0, "Invalid WL parameters");

    DeviceBuffer d_init_spins, d_present;
    InitArgs ia{};
    if (c.initial_spins) {
        std::vector<int8_t> padded(W * ld, 0);
        std::vector<uint8_t> present(W, 1);
        for (uint64_t w = 0; w < W; ++w) {
            if (c.initial_spins_present && !c.initial_spins_present[w]) {
                present[w] = 0;
                continue;
            }
            for (uint64_t i = 0; i < n; ++i) {
                const int8_t sp = c.initial_spins[w * n + i];
                if (sp != -1 && sp != 1) ctor_failure(w, "Spins must be +/-1");
                padded[w * ld + i] = sp;
            }
        }
        d_init_spins.allocate(padded.size());
        d_present.allocate(W);
        check_cuda(cudaMemcpyAsync(d_init_spins.ptr, padded.data(), padded.size(), cudaMemcpyHostToDevice, stream_),
                   "copy spins");
        check_cuda(cudaMemcpyAsync(d_present.ptr, present.data(), W, cudaMemcpyHostToDevice, stream_), "copy");
        ia.initial_spins = d_init_spins.get<int8_t>();
        ia.present = d_present.get<uint8_t>();
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }
    DeviceBuffer d_reports(W * sizeof(InitReport));
    ia.reports = d_reports.get<InitReport>();
    ia.init_max_attempts = c.wl.initialization_max_attempts;
    ia.target_fraction = c.wl.initialization_target_fraction;
    ia.temperature_fraction = c.wl.initialization_temperature_fraction;
    ia.stall_per_spin = c.wl.initialization_stall_attempts_per_spin;
    ia.temperature_multiplier = c.wl.initialization_temperature_multiplier;
    ia.max_temperature_fraction = c.wl.initialization_max_temperature_fraction;
    ia.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(v, smem_fields_, features_));
    launch_init(v, ia, 1, stream_);
    std::vector<InitReport> reports(W);
    check_cuda(cudaMemcpyAsync(reports.data(), d_reports.ptr, W * sizeof(InitReport), cudaMemcpyDeviceToHost, stream_),
               "copy reports");
    check_cuda(cudaStreamSynchronize(stream_), "init");
    for (uint64_t w = 0; w < W; ++w) {
        const InitReport& r = reports[w];
        if (r.status == 0) continue;
        const uint64_t b = win_[2 * (w / wpw_)], e = win_[2 * (w / wpw_) + 1];
        const double lower = c.emin + static_cast<double>(b) * c.bin_width;
        const double upper = c.emin + static_cast<double>(e) * c.bin_width;
        std::ostringstream m;
        m.precision(17);
        m << "Target Metropolis initialization did not reach target band [" << r.target - r.half_width << ", "
          << r.target + r.half_width << "] for energy window bins [" << b << ", " << e << "), energy bounds ["
          << lower << ", " << upper << (e == bins_ ? ']' : ')') << " after " << c.wl.initialization_max_attempts
          << " attempts; reached energy range [" << r.minimum_reached << ", " << r.maximum_reached
          << "], closest energy " << r.closest;
        const int64_t cb = grid_index(grid_, r.closest);
        if (cb >= 0) m << " (bin " << cb << ')';
        else m << " (outside the energy grid)";
        m << ", distance to target band " << std::max(0.0, r.closest_distance - r.half_width)
          << "; adaptive search used " << r.increases << " temperature increases up to " << r.highest_temperature
          << " and " << r.restarts << " random restarts (stall interval " << r.stall << " attempts)";
        ctor_failure(w, m.str());
    }

    // multi-walker checkpoint (an extension: the reference checkpoints 1 x 1 runs only)
    checkpointing_all_ = !checkpoint_path_.empty() && W > 1;
    if (checkpointing_all_) {
        std::ifstream probe(checkpoint_path_, std::ios::binary);
        if (probe) {
            probe.close();
            try {
                load_run(checkpoint_path_);
            } catch (const std::exception& e) {
                std::cerr << "warning: run checkpoint was not restored: " << e.what() << "; starting a new run\n";
            }
        }
    }

    // single-walker checkpoint restore (src/parallel.cpp:354-360)
    checkpointing_ = !checkpoint_path_.empty() && windows_ == 1 && wpw_ == 1;
    if (checkpointing_) {
        std::vector<int8_t> sp;
        std::vector<double> fl, lg;
        std::vector<uint64_t> hs;
        std::vector<uint8_t> ac;
        wlg_snapshot s{};
        std::string error;
        try {
            if (!load_checkpoint_file(checkpoint_path_, sp, fl, lg, hs, ac, s, error)) throw WlgError(WLG_ERR_IO, error);
            if (sp.size() != n || fl.size() != n || lg.size() != B || hs.size() != B || ac.size() != B)
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Checkpoint is incompatible with walker");
            s.spins = sp.data();
            s.fields = fl.data();
            s.log_g = lg.data();
            s.histogram = hs.data();
            s.active = ac.data();
            restore(0, s);
        } catch (const std::exception& e) {
            std::cerr << "warning: checkpoint was not restored: " << e.what() << "; starting a new run\n";
        }
    }
    next_progress_ = now_seconds() + c.progress_interval_seconds;
}

std::vector<WalkerState> Engine::download_states() {
    std::vector<WalkerState> s(walkers_);
    check_cuda(cudaMemcpyAsync(s.data(), d_ws_.ptr, walkers_ * sizeof(WalkerState), cudaMemcpyDeviceToHost, stream_),
               "copy states");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    return s;
}

void Engine::check_device_error() {
    Control ctl{};
    check_cuda(cudaMemcpyAsync(&ctl, d_ctl_.ptr, sizeof ctl, cudaMemcpyDeviceToHost, stream_), "copy control");
    check_cuda(cudaStreamSynchronize(stream_), "epoch");
    done_ = ctl.done != 0;
    epochs_ = ctl.epoch;
    if (ctl.error == WLG_ERR_ESCAPED) throw WlgError(WLG_ERR_ESCAPED, "Walker escaped its energy window");
    if (ctl.error == WLG_ERR_TIMEOUT)
        throw WlgError(WLG_ERR_TIMEOUT, "A bounded device wait gave up (walker " + std::to_string(ctl.error_walker) +
                                            "); the walker's state was not written back");
    if (ctl.error) throw WlgError(static_cast<wlg_status>(ctl.error), "device error");
}

void Engine::inject_wait_timeout() {
    view_.p.withhold_draws = 1;
    // the epoch graph holds the kernels' arguments by value: capture it again
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
}

void Engine::build_graph() {
    if (graph_exec_) return;
    WalkArgs a{};
    a.first = 0;
    a.count = static_cast<int32_t>(walkers_);
    a.fixed_batch = 0;
    a.epoch_mode = 1;
    a.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(view_, smem_fields_, features_));
    // make sure the kernel attributes are set before capture
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        for (int e = 0; e < epochs_per_graph; ++e) launch_epoch(a);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(stream_, &graph_), "end capture");
    check_cuda(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
    graph_epochs_ = epochs_per_graph;
}

void Engine::launch_epochs(uint64_t count) {
    if (window_sweep_) {  // every epoch of the chunk in one launch, no graph
        while (count > 0) {
            const uint32_t e = static_cast<uint32_t>(std::min<uint64_t>(count, 1u << 30));
            launch_sweep_window(view_, e, stream_);
            count -= e;
        }
        return;
    }
    WalkArgs a{};
    a.first = 0;
    a.count = static_cast<int32_t>(walkers_);
    a.fixed_batch = 0;
    a.epoch_mode = 1;
    a.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(view_, smem_fields_, features_));
    if (count == static_cast<uint64_t>(epochs_per_graph) && epochs_per_graph > 1) {
        // first use primes the kernel attributes outside of capture
        if (!graph_exec_) {
            launch_epoch(a);
            count -= 1;
            build_graph();
            for (uint64_t e = 0; e < count; ++e) launch_epoch(a);
            return;
        }
        check_cuda(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
        return;
    }
    for (uint64_t e = 0; e < count; ++e) launch_epoch(a);
}

void Engine::maybe_checkpoint() {
    if (checkpointing_all_) {
        WalkerState st{};
        check_cuda(cudaMemcpyAsync(&st, d_ws_.ptr, sizeof st, cudaMemcpyDeviceToHost, stream_), "copy state");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        if (st.attempted - last_checkpoint_ >= cfg_.checkpoint_interval_attempts) {
            save_run(checkpoint_path_);
            last_checkpoint_ = st.attempted;
        }
        return;
    }
    if (!checkpointing_) return;
    WalkerState st{};
    check_cuda(cudaMemcpyAsync(&st, d_ws_.ptr, sizeof st, cudaMemcpyDeviceToHost, stream_), "copy state");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    if (st.attempted - last_checkpoint_ >= cfg_.checkpoint_interval_attempts) {
        std::vector<int8_t> sp(sys_.n);
        std::vector<double> fl(sys_.n), lg(bins_);
        std::vector<uint64_t> hs(bins_);
        std::vector<uint8_t> ac(bins_);
        wlg_snapshot s{};
        s.spins = sp.data();
        s.fields = fl.data();
        s.log_g = lg.data();
        s.histogram = hs.data();
        s.active = ac.data();
        snapshot(0, &s);
        save_checkpoint_file(checkpoint_path_, s, sys_.n, bins_);
        last_checkpoint_ = st.attempted;
    }
}

void Engine::print_progress(bool final_line) {
    if (cfg_.progress_interval_seconds <= 0.0) return;
    if (final_line) {
        if (progress_width_ != 0) std::cout << '\n' << std::flush;
        return;
    }
    if (now_seconds() < next_progress_) return;
    const auto states = download_states();
    uint64_t attempted = 0;
    double factor = 0.0, flatness = 1.0;
    uint64_t stages[3] = {0, 0, 0};
    for (uint64_t w = 0; w < windows_; ++w) attempted = std::max(attempted, states[w * wpw_].attempted);
    for (const auto& s : states) {
        factor = std::max(factor, s.factor);
        ++stages[s.stage == kWangLandau ? 0 : s.stage == kInverseTime ? 1 : 2];
        if (s.stage == kWangLandau) flatness = std::min(flatness, s.last_flatness);
    }
    std::ostringstream line;
    line << "progress mcs=" << static_cast<double>(attempted) / static_cast<double>(sys_.n)
         << " attempted_flips_per_walker=" << attempted << (p_.inverse_time ? " coverage=" : " flatness=") << flatness
         << " factor=" << factor << " stages=" << stages[0] << '/' << stages[1] << '/' << stages[2];
    const std::string text = line.str();
    std::cout << '\r' << text;
    if (progress_width_ > text.size()) std::cout << std::string(progress_width_ - text.size(), ' ');
    std::cout << std::flush;
    progress_width_ = std::max(progress_width_, text.size());
    next_progress_ = now_seconds() + cfg_.progress_interval_seconds;
}

void Engine::run_epochs(uint64_t max_epochs, uint64_t* epochs_run, int32_t* done) {
    const uint64_t start = epochs_;
    uint64_t budget = max_epochs;
    while (!done_ && budget > 0) {
        // the single-window kernel runs about a million attempts per walker per launch
        const uint64_t per_launch =
            window_sweep_ ? std::clamp<uint64_t>((uint64_t{1} << 20) / std::max<uint64_t>(1, p_.exchange_interval), 1, 4096)
                          : static_cast<uint64_t>(epochs_per_graph);
        uint64_t chunk = std::min<uint64_t>(budget, per_launch);
        if (checkpointing_) {
            WalkerState st{};
            check_cuda(cudaMemcpyAsync(&st, d_ws_.ptr, sizeof st, cudaMemcpyDeviceToHost, stream_), "copy state");
            check_cuda(cudaStreamSynchronize(stream_), "sync");
            const uint64_t since = st.attempted - last_checkpoint_;
            const uint64_t need = cfg_.checkpoint_interval_attempts > since ? cfg_.checkpoint_interval_attempts - since : 0;
            const uint64_t epochs_needed = std::max<uint64_t>(1, (need + p_.exchange_interval - 1) / p_.exchange_interval);
            chunk = std::min(chunk, epochs_needed);
        }
        if (recompute_epochs_ > 1) chunk = std::min(chunk, std::max<uint64_t>(1, next_recompute_ - epochs_));
        launch_epochs(chunk);
        budget -= std::min(budget, chunk);
        after_epochs();
    }
    if (done_) finish();
    if (epochs_run) *epochs_run = epochs_ - start;
    if (done) *done = done_ ? 1 : 0;
}

// The FP64 recompute of a mixed-precision run: all configurations' fields and energies from
// the FP64 J (reference summation order), then the per-walker drift measurement and resync.
// Stream-ordered, no host synchronisation: a recompute every epoch is part of the epoch graph.
void Engine::launch_recompute() {
    compute_fields(view_, d_spins_.get<int8_t>(), static_cast<int64_t>(sys_.ld), d_rfields_.get<double>(),
                   static_cast<int64_t>(sys_.ld), d_renergy_.get<double>(), static_cast<int>(walkers_), stream_);
    launch_resync(view_, d_rfields_.get<double>(), d_renergy_.get<double>(), d_prec_.get<PrecisionReport>(),
                  stream_);
}

void Engine::recompute_fields() {
    launch_recompute();
    check_device_error();
}

// One epoch of run_rewl on the stream: the sweep, the exchange and, when the recompute
// interval is one epoch, the FP64 recompute.
void Engine::launch_epoch(const WalkArgs& a) {
    if (window_sweep_) {
        launch_sweep_window(view_, 1, stream_);
        return;
    }
    launch_walk(view_, a, walkers_per_block, stream_);
    launch_exchange(view_, stream_);
    if (recompute_epochs_ == 1) launch_recompute();
}

void Engine::precision_report(wlg_precision_report* out) {
    PrecisionReport r{};
    check_cuda(cudaMemcpyAsync(&r, d_prec_.ptr, sizeof r, cudaMemcpyDeviceToHost, stream_), "copy report");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    *out = wlg_precision_report{};
    out->coupling_precision = precision_;
    out->recompute_interval_attempts = recompute_epochs_ ? cfg_.recompute_interval_attempts : 0;
    out->recomputes = r.recomputes;
    out->resynced = r.resynced;
    out->deferred = r.deferred;
    out->bin_changes = r.bin_changes;
    std::memcpy(&out->max_field_drift, &r.max_field_drift_bits, sizeof(double));
    std::memcpy(&out->max_energy_drift, &r.max_energy_drift_bits, sizeof(double));
}

// Host work between launches: device errors, the mixed-precision recompute, the checkpoint
// and the progress line.
void Engine::after_epochs() {
    check_device_error();
    if (recompute_epochs_ > 1 && !done_ && epochs_ >= next_recompute_) {
        recompute_fields();
        next_recompute_ = epochs_ + recompute_epochs_;
    }
    maybe_checkpoint();
    print_progress(false);
}

// Once, when the run has terminated: the representatives still pending and the final line.
void Engine::finish() {
    if (finished_) return;
    finished_ = true;
    if (p_.collect) launch_flush_pending(view_, stream_);
    print_progress(true);
}

cudaGraph_t Engine::epoch_graph() {
    if (!graph_exec_) {
        WalkArgs a{};
        a.first = 0;
        a.count = static_cast<int32_t>(walkers_);
        a.epoch_mode = 1;
        a.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(view_, smem_fields_, features_));
        launch_epoch(a);  // sets the kernel attributes
        after_epochs();
        build_graph();
    }
    return graph_;
}

void Engine::after_external_epochs() {
    after_epochs();
    if (done_) finish();
}

Batch::Batch(const std::vector<Engine*>& engines) : engines_(engines) {
    if (engines_.empty()) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "an empty batch");
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    for (size_t i = 0; i < engines_.size(); ++i) {
        if (!engines_[i]) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "null engine in a batch");
        if (engines_[i]->device != device)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "every engine of a batch must live on the current device");
        for (size_t j = 0; j < i; ++j)
            if (engines_[j] == engines_[i]) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "an engine appears twice");
    }
    check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaGraphCreate(&graph_, 0), "cudaGraphCreate");
    for (Engine* e : engines_) {
        cudaGraphNode_t node = nullptr;
        check_cuda(cudaGraphAddChildGraphNode(&node, graph_, nullptr, 0, e->epoch_graph()), "child graph");
        epochs_per_launch_ = std::max<uint64_t>(epochs_per_launch_, static_cast<uint64_t>(e->epochs_per_graph));
    }
    check_cuda(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate");
}

Batch::~Batch() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Batch::run_epochs(uint64_t max_epochs, uint64_t* launches, int32_t* all_done) {
    uint64_t budget = max_epochs, n = 0;
    auto everyone_done = [&] {
        for (Engine* e : engines_)
            if (!e->is_done()) return false;
        return true;
    };
    while (budget > 0 && !everyone_done()) {
        check_cuda(cudaGraphLaunch(exec_, stream_), "graph launch");
        check_cuda(cudaStreamSynchronize(stream_), "batch");
        ++n;
        for (Engine* e : engines_) e->after_external_epochs();
        budget -= std::min(budget, epochs_per_launch_);
    }
    if (launches) *launches = n;
    if (all_done) *all_done = everyone_done() ? 1 : 0;
}

void Engine::run(wlg_run_totals* out) {
    while (!done_) run_epochs(~0ULL, nullptr, nullptr);
    if (out) totals(out);
}

// The product path (run_epochs: CUDA-graph replays and the host's checks between them) with
// one CUDA event before and one after, on the engine's stream.
void Engine::time_run(uint64_t epochs, wlg_epoch_timing* out) {
    wlg_run_totals before{}, after{};
    totals(&before);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    try {
        const uint64_t start = epochs_;
        check_cuda(cudaEventRecord(e0, stream_), "record");
        run_epochs(epochs, nullptr, nullptr);
        check_cuda(cudaEventRecord(e1, stream_), "record");
        check_cuda(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        totals(&after);
        *out = wlg_epoch_timing{};
        out->epochs = epochs_ - start;
        out->total_ms = ms;
        out->attempted = after.attempted - before.attempted;
        out->accepted = after.accepted - before.accepted;
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

void Engine::time_epochs(uint64_t epochs, wlg_epoch_timing* out) {
    wlg_run_totals before{}, after{};
    totals(&before);
    WalkArgs a{};
    a.first = 0;
    a.count = static_cast<int32_t>(walkers_);
    a.epoch_mode = 1;
    a.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(view_, smem_fields_, features_));
    std::vector<cudaEvent_t> ev(3 * epochs + 1);
    for (auto& e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
    uint64_t ran = 0;
    try {
        check_cuda(cudaEventRecord(ev[0], stream_), "record");
        for (uint64_t k = 0; k < epochs && !done_; ++k) {
            launch_walk(view_, a, walkers_per_block, stream_);
            check_cuda(cudaEventRecord(ev[3 * k + 1], stream_), "record");
            launch_exchange(view_, stream_);
            check_cuda(cudaEventRecord(ev[3 * k + 2], stream_), "record");
            if (recompute_epochs_ == 1) launch_recompute();
            check_cuda(cudaEventRecord(ev[3 * k + 3], stream_), "record");
            ++ran;
        }
        check_device_error();
        wlg_epoch_timing t{};
        t.epochs = ran;
        for (uint64_t k = 0; k < ran; ++k) {
            float walk = 0.f, ex = 0.f;
            check_cuda(cudaEventElapsedTime(&walk, ev[3 * k], ev[3 * k + 1]), "elapsed");
            check_cuda(cudaEventElapsedTime(&ex, ev[3 * k + 1], ev[3 * k + 2]), "elapsed");
            t.walk_ms += walk;
            t.exchange_ms += ex;
        }
        float total = 0.f;
        if (ran) check_cuda(cudaEventElapsedTime(&total, ev[0], ev[3 * ran]), "elapsed");
        t.total_ms = total;
        totals(&after);
        t.attempted = after.attempted - before.attempted;
        t.accepted = after.accepted - before.accepted;
        *out = t;
    } catch (...) {
        for (auto& e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto& e : ev) cudaEventDestroy(e);
}

void Engine::set_launch(int wpb, int epg) {
    if (wpb < 0 || wpb > 8 || epg < 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "invalid launch shape");
    if (wpb) walkers_per_block = wpb;
    if (epg && epg != epochs_per_graph) {
        epochs_per_graph = epg;
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (graph_) cudaGraphDestroy(graph_);
        graph_exec_ = nullptr;
        graph_ = nullptr;
    }
    if (wpb && graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        cudaGraphDestroy(graph_);
        graph_exec_ = nullptr;
        graph_ = nullptr;
    }
}

// Launch-shape autotuner: each candidate (staging ring of the split sweep, walkers per CTA of
// the generic sweep, epochs per graph replay) runs `trial_epochs` real epochs of this engine
// through the product path after a warm-up replay that builds its graph, timed with device
// events; the fastest per epoch is kept.  The candidates are timed twice, in order and then in
// reverse order, and each one's two times are added: the cost of an epoch drifts as the run
// moves on (acceptance, stage), and a drift that is linear over the trials adds the same to
// every candidate's sum.  The launch shape never changes results, so the trial epochs are
// ordinary epochs of the run.  (The exchange interval, which does change the sampled
// trajectories, is left as configured.)
void Engine::autotune(uint64_t trial_epochs, wlg_autotune_report* out) {
    if (trial_epochs == 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "autotune needs at least one trial epoch");
    const bool generic = sys_.csr || sys_.ld > 1024 || features_;
    const int wpbs_generic[] = {1, 2, 4, 8};
    const int wpbs_dense[] = {1};
    const int* wpbs = generic ? wpbs_generic : wpbs_dense;
    const int n_wpb = generic ? 4 : 1;
    const int epgs[] = {4, 8, 16, 32, 64};
    // the split sweep's staging depth (16 or 32 draws with their J rows) where it serves the engine
    std::vector<int> rings;
    for (int rl : split_ring_logs(view_)) rings.push_back(1 << rl);
    if (rings.empty()) rings.push_back(0);
    struct Candidate {
        int ring, wpb, epg;
        double ms = 0.0;  // per epoch, summed over the passes
        int passes = 0;
    };
    std::vector<Candidate> cands;
    for (int ring : rings)
        for (int a = 0; a < n_wpb; ++a)
            for (int epg : epgs) cands.push_back({ring, wpbs[a], epg});
    wlg_autotune_report r{};
    for (int pass = 0; pass < 2; ++pass) {
        for (size_t k = 0; k < cands.size() && !done_; ++k) {
            Candidate& c = cands[pass == 0 ? k : cands.size() - 1 - k];
            if (c.ring) set_staging_ring(c.ring);
            set_launch(c.wpb, c.epg);
            wlg_epoch_timing t{};
            time_run(static_cast<uint64_t>(c.epg), &t);  // builds and warms the graph
            const uint64_t rounds = std::max<uint64_t>(1, (trial_epochs + c.epg - 1) / c.epg);
            time_run(rounds * c.epg, &t);
            ++r.trials;
            if (t.epochs == 0) continue;
            c.ms += t.total_ms / static_cast<double>(t.epochs);
            ++c.passes;
        }
    }
    double best = std::numeric_limits<double>::infinity();
    int best_wpb = walkers_per_block, best_epg = epochs_per_graph, best_ring = staging_ring();
    const int most = std::max_element(cands.begin(), cands.end(), [](const Candidate& x, const Candidate& y) {
                         return x.passes < y.passes;
                     })->passes;
    for (const Candidate& c : cands) {
        if (c.passes == 0 || c.passes < most) continue;  // a run that ended during the trials
        if (c.ms < best) {
            best = c.ms;
            best_wpb = c.wpb;
            best_epg = c.epg;
            best_ring = c.ring ? c.ring : staging_ring();
        }
    }
    if (std::isfinite(best)) best /= most;
    if (rings.front() != 0) set_staging_ring(best_ring);
    set_launch(best_wpb, best_epg);
    r.walkers_per_block = best_wpb;
    r.epochs_per_graph = best_epg;
    r.ms_per_epoch = std::isfinite(best) ? best : 0.0;
    r.staging_ring = staging_ring();
    if (out) *out = r;
}

void Engine::set_staging_ring(int entries) {
    int rl = 0;
    if (entries == 16) rl = 4;
    else if (entries == 32) rl = 5;
    else if (entries != 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "The staging ring holds 16 or 32 draws");
    if (rl != 0) {
        const std::vector<int> ok = split_ring_logs(view_);
        if (std::find(ok.begin(), ok.end(), rl) == ok.end())
            throw WlgError(WLG_ERR_INVALID_ARGUMENT,
                           "This engine's sweep has no staging ring of " + std::to_string(entries) + " draws");
    }
    if (rl == view_.split_ring_log) return;
    view_.split_ring_log = rl;
    // the epoch graph holds the kernels' arguments by value: capture it again
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
}

int Engine::staging_ring() const {
    if (split_ring_logs(view_).empty()) return 0;
    return 1 << (view_.split_ring_log == 5 ? 5 : 4);
}

void Engine::totals(wlg_run_totals* out) {
    Control ctl{};
    check_cuda(cudaMemcpyAsync(&ctl, d_ctl_.ptr, sizeof ctl, cudaMemcpyDeviceToHost, stream_), "copy control");
    const auto states = download_states();
    wlg_run_totals t{};
    t.converged = 1;
    for (const auto& s : states) {
        t.attempted += s.attempted;
        t.accepted += s.accepted;
        t.forced_accepted += s.forced;
        t.converged &= s.stage == kFrozen ? 1 : 0;
    }
    t.exchange_attempted = ctl.exchange_attempted;
    t.exchange_accepted = ctl.exchange_accepted;
    t.epochs = ctl.epoch;
    *out = t;
}

void Engine::window(uint64_t w, uint64_t* begin, uint64_t* end) const {
    if (w >= windows_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "window index out of range");
    *begin = win_[2 * w];
    *end = win_[2 * w + 1];
}

void Engine::fragment(uint64_t w, int allow_empty, double* log_g, uint64_t* hist, double* sem, uint8_t* valid) {
    if (w >= windows_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "window index out of range");
    const size_t B = bins_;
    char* base = d_scratch_.get<char>();
    double* d_lg = reinterpret_cast<double*>(base);
    uint64_t* d_h = reinterpret_cast<uint64_t*>(base + 8 * B);
    double* d_se = reinterpret_cast<double*>(base + 16 * B);
    uint8_t* d_v = reinterpret_cast<uint8_t*>(base + 24 * B);
    int* d_status = reinterpret_cast<int*>(base + ((25 * B + 15) / 16) * 16);
    launch_summarize(view_, static_cast<int>(w), 1, allow_empty, d_lg, d_h, d_se, d_v, d_status, stream_);
    int status = 0;
    check_cuda(cudaMemcpyAsync(log_g, d_lg, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(hist, d_h, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(sem, d_se, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(valid, d_v, B, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "summarize");
    if (status) throw WlgError(WLG_ERR_RUNTIME, "Walkers in an energy window have no common active bin");
}

void Engine::fragments(int allow_empty, double* log_g, uint64_t* hist, double* sem, uint8_t* valid) {
    const size_t WB = windows_ * bins_;
    const size_t status_at = ((25 * WB + 15) / 16) * 16;
    if (!d_frag_.ptr) d_frag_.allocate(status_at + 4 * windows_);
    char* base = d_frag_.get<char>();
    double* d_lg = reinterpret_cast<double*>(base);
    uint64_t* d_h = reinterpret_cast<uint64_t*>(base + 8 * WB);
    double* d_se = reinterpret_cast<double*>(base + 16 * WB);
    uint8_t* d_v = reinterpret_cast<uint8_t*>(base + 24 * WB);
    int* d_status = reinterpret_cast<int*>(base + status_at);
    launch_summarize(view_, 0, static_cast<int>(windows_), allow_empty, d_lg, d_h, d_se, d_v, d_status, stream_);
    std::vector<int> status(windows_, 0);
    check_cuda(cudaMemcpyAsync(log_g, d_lg, WB * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(hist, d_h, WB * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(sem, d_se, WB * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(valid, d_v, WB, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(status.data(), d_status, 4 * windows_, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "summarize");
    for (int st : status)
        if (st) throw WlgError(WLG_ERR_RUNTIME, "Walkers in an energy window have no common active bin");
}

void Engine::stitch(int complete_range, double* log_g, uint64_t* hist, double* sem, uint8_t* valid,
                    wlg_join_quality* joins, int32_t* fully_normalized) {
    const size_t WB = windows_ * bins_, B = bins_;
    const size_t status_at = ((25 * WB + 15) / 16) * 16;
    if (!d_frag_.ptr) d_frag_.allocate(status_at + 4 * windows_);
    char* base = d_frag_.get<char>();
    double* d_lg = reinterpret_cast<double*>(base);
    uint64_t* d_h = reinterpret_cast<uint64_t*>(base + 8 * WB);
    double* d_se = reinterpret_cast<double*>(base + 16 * WB);
    uint8_t* d_v = reinterpret_cast<uint8_t*>(base + 24 * WB);
    int* d_status = reinterpret_cast<int*>(base + status_at);
    // the stitched arrays, the joins and the status word
    const size_t joins_at = ((25 * B + 15) / 16) * 16;
    const size_t stitch_status_at = joins_at + sizeof(wlg_join_quality) * windows_;
    if (!d_stitch_.ptr) d_stitch_.allocate(stitch_status_at + 16);
    char* out = d_stitch_.get<char>();
    double* o_lg = reinterpret_cast<double*>(out);
    uint64_t* o_h = reinterpret_cast<uint64_t*>(out + 8 * B);
    double* o_se = reinterpret_cast<double*>(out + 16 * B);
    uint8_t* o_v = reinterpret_cast<uint8_t*>(out + 24 * B);
    wlg_join_quality* o_j = reinterpret_cast<wlg_join_quality*>(out + joins_at);
    int* o_status = reinterpret_cast<int*>(out + stitch_status_at);
    launch_summarize(view_, 0, static_cast<int>(windows_), 0, d_lg, d_h, d_se, d_v, d_status, stream_);
    launch_stitch(static_cast<int>(windows_), static_cast<int>(B), view_.win_begin, view_.win_end, d_lg, d_h, d_se, d_v,
                  d_status, cfg_.bin_width, complete_range, o_lg, o_h, o_se, o_v, o_j, o_status, stream_);
    int status = 0;
    std::vector<wlg_join_quality> q(windows_ > 1 ? windows_ - 1 : 0);
    check_cuda(cudaMemcpyAsync(log_g, o_lg, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(hist, o_h, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(sem, o_se, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(valid, o_v, B, cudaMemcpyDeviceToHost, stream_), "copy");
    if (!q.empty())
        check_cuda(cudaMemcpyAsync(q.data(), o_j, q.size() * sizeof(wlg_join_quality), cudaMemcpyDeviceToHost, stream_),
                   "copy");
    check_cuda(cudaMemcpyAsync(&status, o_status, sizeof status, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "stitch");
    switch (status) {
        case 0: break;
        case kStitchNoCommonBin: throw WlgError(WLG_ERR_RUNTIME, "Walkers in an energy window have no common active bin");
        case kStitchNoOverlap:
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "DOS fragments must overlap and match the global grid");
        case kStitchNoCommonOverlapBin:
            throw WlgError(WLG_ERR_RUNTIME, "Adjacent DOS fragments have no common valid overlap bin");
        case kStitchIncomplete:
            throw WlgError(WLG_ERR_RUNTIME, "Complete-range normalization requires every DOS bin to be valid");
        case kStitchNoValidBins: throw WlgError(WLG_ERR_RUNTIME, "Stitched DOS has no valid bins");
        default: throw WlgError(WLG_ERR_DEVICE, "stitch_kernel failed");
    }
    if (complete_range) {
        // N ln 2 - log sum exp, with the C library's exp and log (as the reference computes it)
        double top = -std::numeric_limits<double>::infinity();
        for (size_t i = 0; i < B; ++i)
            if (std::isfinite(log_g[i])) top = std::max(top, log_g[i]);
        double sum = 0.0;
        for (size_t i = 0; i < B; ++i)
            if (std::isfinite(log_g[i])) sum += std::exp(log_g[i] - top);
        const double shift = static_cast<double>(sys_.n) * std::log(2.0) - (top + std::log(sum));
        for (size_t i = 0; i < B; ++i)
            if (valid[i] != 0) log_g[i] += shift;
    }
    if (joins) std::copy(q.begin(), q.end(), joins);
    if (fully_normalized) *fully_normalized = complete_range ? 1 : 0;
}

void Engine::sampling(uint64_t w, double* sq, uint64_t* samples, uint64_t* round_trips, uint64_t* walkers) {
    if (w >= windows_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "window index out of range");
    if (!p_.collect) throw WlgError(WLG_ERR_LOGIC, "window statistics were not collected");
    const size_t B = bins_;
    char* base = d_scratch_.get<char>();
    double* d_sq = reinterpret_cast<double*>(base);
    uint64_t* d_ds = reinterpret_cast<uint64_t*>(base + 8 * B);
    uint64_t* d_t = reinterpret_cast<uint64_t*>(base + 16 * B);
    launch_sampling(view_, static_cast<int>(w), d_sq, d_ds, d_t, stream_);
    check_cuda(cudaMemcpyAsync(sq, d_sq, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(samples, d_ds, B * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(round_trips, d_t, 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "sampling");
    *walkers = wpw_;
}

void Engine::walker_statistics(wlg_walker_statistics* out, uint64_t capacity) {
    if (capacity < walkers_) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "walker statistics buffer too small");
    auto* d_out = d_scratch_.get<wlg_walker_statistics>();
    launch_walker_statistics(view_, d_out, stream_);
    check_cuda(cudaMemcpyAsync(out, d_out, walkers_ * sizeof(wlg_walker_statistics), cudaMemcpyDeviceToHost, stream_),
               "copy");
    check_cuda(cudaStreamSynchronize(stream_), "statistics");
}

void Engine::representatives(double* energies, int8_t* spins, uint64_t capacity, uint64_t* count) {
    *count = 0;
    if (!p_.collect) return;
    launch_flush_pending(view_, stream_);
    const uint64_t R = walkers_ * kRepresentatives;
    std::vector<double> e(R);
    std::vector<uint8_t> present(R);
    std::vector<int8_t> s(R * sys_.ld);
    check_cuda(cudaMemcpyAsync(e.data(), d_rep_energy_.ptr, R * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(present.data(), d_rep_present_.ptr, R, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(s.data(), d_rep_spins_.ptr, R * sys_.ld, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    uint64_t k = 0;
    for (uint64_t q = 0; q < R; ++q) {
        if (!present[q]) continue;
        if (k < capacity) {
            if (energies) energies[k] = e[q];
            if (spins) std::memcpy(spins + k * sys_.n, s.data() + q * sys_.ld, sys_.n);
        }
        ++k;
    }
    *count = k;
}

void Engine::run_attempts(uint64_t walker, uint64_t count) {
    if (walker >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    if (count == 0) return;
    WalkArgs a{};
    a.first = static_cast<int32_t>(walker);
    a.count = 1;
    a.fixed_batch = count;
    a.epoch_mode = 0;
    a.smem_per_walker = static_cast<int32_t>(walker_smem_bytes(view_, smem_fields_, features_));
    Control ctl{};
    check_cuda(cudaMemcpyAsync(&ctl, d_ctl_.ptr, sizeof ctl, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    launch_walk(view_, a, 1, stream_);
    Control after{};
    check_cuda(cudaMemcpyAsync(&after, d_ctl_.ptr, sizeof after, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "run_attempts");
    if (after.error && !ctl.error) {
        const int err = after.error;
        after.error = 0;
        after.done = ctl.done;
        check_cuda(cudaMemcpyAsync(d_ctl_.ptr, &after, sizeof after, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        if (err == WLG_ERR_ESCAPED) throw WlgError(WLG_ERR_ESCAPED, "Walker escaped its energy window");
        throw WlgError(static_cast<wlg_status>(err), "device error");
    }
}

void Engine::snapshot(uint64_t walker, wlg_snapshot* out) {
    if (walker >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    WalkerState st{};
    check_cuda(cudaMemcpyAsync(&st, d_ws_.get<WalkerState>() + walker, sizeof st, cudaMemcpyDeviceToHost, stream_),
               "copy");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    const size_t off = walker * bins_;
    if (out->spins)
        check_cuda(cudaMemcpyAsync(out->spins, d_spins_.get<int8_t>() + static_cast<size_t>(st.slot) * sys_.ld, sys_.n,
                                   cudaMemcpyDeviceToHost, stream_), "copy");
    if (out->fields)
        check_cuda(cudaMemcpyAsync(out->fields, d_fields_.get<double>() + static_cast<size_t>(st.slot) * sys_.ld,
                                   sys_.n * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    if (out->log_g)
        check_cuda(cudaMemcpyAsync(out->log_g, d_log_g_.get<double>() + off, bins_ * 8, cudaMemcpyDeviceToHost, stream_),
                   "copy");
    if (out->histogram)
        check_cuda(cudaMemcpyAsync(out->histogram, d_hist_.get<uint64_t>() + off, bins_ * 8, cudaMemcpyDeviceToHost,
                                   stream_), "copy");
    if (out->active)
        check_cuda(cudaMemcpyAsync(out->active, d_active_.get<uint8_t>() + off, bins_, cudaMemcpyDeviceToHost, stream_),
                   "copy");
    check_cuda(cudaStreamSynchronize(stream_), "snapshot");
    out->walker_id = walker;
    out->energy = st.energy;
    out->factor = st.factor;
    out->attempted = st.attempted;
    out->accepted = st.accepted;
    out->forced_accepted = st.forced;
    out->last_accepted_attempt = st.last_accepted;
    out->stage = static_cast<uint8_t>(st.stage);
    for (int k = 0; k < 4; ++k) out->rng_state[k] = st.rng[k];
}

// restore (src/wang_landau.cpp:420-466).  As in the reference, the state is replaced before
// the energy / field consistency test, and that test's failure is reported afterwards.
void Engine::restore(uint64_t walker, const wlg_snapshot& s) {
    if (walker >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    if (s.walker_id != walker || !s.spins || !s.fields || !s.log_g || !s.histogram || !s.active)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Checkpoint is incompatible with walker");
    if (s.last_accepted_attempt > s.attempted)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Checkpoint has an invalid last accepted attempt");
    if (s.forced_accepted > s.accepted)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Checkpoint has an invalid forced acceptance count");
    if (!p_.inverse_time && s.stage == WLG_STAGE_INVERSE_TIME)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Checkpoint uses disabled inverse-time refinement");
    WalkerState st{};
    check_cuda(cudaMemcpyAsync(&st, d_ws_.get<WalkerState>() + walker, sizeof st, cudaMemcpyDeviceToHost, stream_),
               "copy");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
    const uint64_t n = sys_.n, B = bins_;
    const uint64_t wb = win_[2 * st.window], we = win_[2 * st.window + 1];
    std::vector<uint8_t> active(s.active, s.active + B), refine(B, 0);
    uint64_t active_count = 0, refine_count = 0;
    for (uint64_t i = wb; i < we; ++i) {
        active[i] = active[i] != 0 ? 1 : 0;
        active_count += active[i];
        if (p_.nalivaiko) {
            refine[i] = s.histogram[i] != 0 ? 1 : 0;
            refine_count += refine[i];
        }
    }
    const size_t off = walker * B;
    std::vector<int8_t> spins(sys_.ld, 0);
    std::vector<double> fields(sys_.ld, 0.0);
    std::memcpy(spins.data(), s.spins, n);
    std::memcpy(fields.data(), s.fields, n * 8);
    check_cuda(cudaMemcpyAsync(d_spins_.get<int8_t>() + static_cast<size_t>(st.slot) * sys_.ld, spins.data(), sys_.ld,
                               cudaMemcpyHostToDevice, stream_), "copy");
    check_cuda(cudaMemcpyAsync(d_fields_.get<double>() + static_cast<size_t>(st.slot) * sys_.ld, fields.data(),
                               sys_.ld * 8, cudaMemcpyHostToDevice, stream_), "copy");
    check_cuda(cudaMemcpyAsync(d_log_g_.get<double>() + off, s.log_g, B * 8, cudaMemcpyHostToDevice, stream_), "copy");
    check_cuda(cudaMemcpyAsync(d_hist_.get<uint64_t>() + off, s.histogram, B * 8, cudaMemcpyHostToDevice, stream_),
               "copy");
    check_cuda(cudaMemcpyAsync(d_active_.get<uint8_t>() + off, active.data(), B, cudaMemcpyHostToDevice, stream_),
               "copy");
    if (features_)
        check_cuda(cudaMemcpyAsync(d_refine_.get<uint8_t>() + off, refine.data(), B, cudaMemcpyHostToDevice, stream_),
                   "copy");
    st.energy = s.energy;
    st.factor = s.factor;
    st.attempted = s.attempted;
    st.accepted = s.accepted;
    st.forced = s.forced_accepted;
    st.last_accepted = s.last_accepted_attempt;
    st.stage = s.stage;
    st.active_count = active_count;
    st.refine_count = refine_count;
    st.last_check = 0;
    for (int k = 0; k < 4; ++k) st.rng[k] = s.rng_state[k];
    const int64_t cb = grid_index(grid_, s.energy);
    st.cur_bin = static_cast<int32_t>(cb);
    if (p_.collect) {
        std::vector<double> zeros(B, 0.0);
        check_cuda(cudaMemcpyAsync(d_sqdisp_.get<double>() + off, zeros.data(), B * 8, cudaMemcpyHostToDevice, stream_),
                   "copy");
        check_cuda(cudaMemsetAsync(d_dsamples_.get<uint64_t>() + off, 0, B * 8, stream_), "memset");
        st.rt_state = 0;
        st.round_trips = 0;
        const double lower = grid_.minimum + static_cast<double>(wb) * grid_.width;
        const double upper = grid_.minimum + static_cast<double>(we) * grid_.width;
        const double margin = p_.round_trip_margin * (upper - lower);
        if (st.energy <= lower + margin) st.rt_state = 1;
        // representatives: every slot is closer than +infinity
        std::vector<double> targets(kRepresentatives), dist(kRepresentatives), energies(kRepresentatives);
        std::vector<uint8_t> present(kRepresentatives, 0);
        check_cuda(cudaMemcpyAsync(targets.data(), d_rep_target_.get<double>() + walker * kRepresentatives,
                                   kRepresentatives * 8, cudaMemcpyDeviceToHost, stream_), "copy");
        check_cuda(cudaMemcpyAsync(energies.data(), d_rep_energy_.get<double>() + walker * kRepresentatives,
                                   kRepresentatives * 8, cudaMemcpyDeviceToHost, stream_), "copy");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        for (int r = 0; r < kRepresentatives; ++r) {
            const double d = std::abs(st.energy - targets[r]);
            if (d < std::numeric_limits<double>::infinity()) {
                dist[r] = d;
                energies[r] = st.energy;
                present[r] = 1;
                check_cuda(cudaMemcpyAsync(d_rep_spins_.get<int8_t>() + (walker * kRepresentatives + r) * sys_.ld,
                                           spins.data(), sys_.ld, cudaMemcpyHostToDevice, stream_), "copy");
            } else {
                dist[r] = std::numeric_limits<double>::infinity();
            }
        }
        check_cuda(cudaMemcpyAsync(d_rep_dist_.get<double>() + walker * kRepresentatives, dist.data(),
                                   kRepresentatives * 8, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaMemcpyAsync(d_rep_energy_.get<double>() + walker * kRepresentatives, energies.data(),
                                   kRepresentatives * 8, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaMemcpyAsync(d_rep_present_.get<uint8_t>() + walker * kRepresentatives, present.data(),
                                   kRepresentatives, cudaMemcpyHostToDevice, stream_), "copy");
        st.rep_pending = 0;
    }
    check_cuda(cudaMemcpyAsync(d_ws_.get<WalkerState>() + walker, &st, sizeof st, cudaMemcpyHostToDevice, stream_),
               "copy");
    // consistency check against a full recompute (src/wang_landau.cpp:459-465)
    DeviceBuffer d_f(sys_.ld * 8), d_e(8);
    compute_fields(view_, d_spins_.get<int8_t>() + static_cast<size_t>(st.slot) * sys_.ld, 0, d_f.get<double>(), 0,
                   d_e.get<double>(), 1, stream_);
    std::vector<double> exact_fields(n);
    double exact = 0.0;
    check_cuda(cudaMemcpyAsync(exact_fields.data(), d_f.ptr, n * 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(&exact, d_e.ptr, 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "restore");
    if (std::abs(exact - s.energy) > 1e-9 * std::max(1.0, std::abs(exact)))
        throw WlgError(WLG_ERR_RUNTIME, "Checkpoint energy does not match spin configuration");
    for (uint64_t i = 0; i < n; ++i)
        if (std::abs(exact_fields[i] - s.fields[i]) > 1e-9 * std::max(1.0, std::abs(exact_fields[i])))
            throw WlgError(WLG_ERR_RUNTIME, "Checkpoint local fields do not match spin configuration");
}

void Engine::histogram_statistics(uint64_t walker, wlg_histogram_statistics* out, int32_t* flags) {
    if (walker >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    char* base = d_scratch_.get<char>();
    auto* d_out = reinterpret_cast<wlg_histogram_statistics*>(base);
    int* d_flags = reinterpret_cast<int*>(base + 128);
    launch_histogram_statistics(view_, static_cast<int>(walker), d_out, d_flags, stream_);
    int f[3] = {0, 0, 0};
    check_cuda(cudaMemcpyAsync(out, d_out, sizeof *out, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaMemcpyAsync(f, d_flags, sizeof f, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "statistics");
    if (flags) for (int k = 0; k < 3; ++k) flags[k] = f[k];
}

void Engine::begin_next_iteration(uint64_t walker) {
    if (walker >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    int* d_status = d_scratch_.get<int>();
    launch_begin_next_iteration(view_, static_cast<int>(walker), d_status, stream_);
    int status = 0;
    check_cuda(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "begin_next_iteration");
    if (status) throw WlgError(WLG_ERR_LOGIC, "WL iteration is not complete");
}

double Engine::exchange_log_probability(uint64_t left, uint64_t right) {
    if (left >= walkers_ || right >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    char* base = d_scratch_.get<char>();
    launch_exchange_pair(view_, static_cast<int>(left), static_cast<int>(right), 0, reinterpret_cast<double*>(base),
                         reinterpret_cast<int*>(base + 16), stream_);
    double lp = 0.0;
    check_cuda(cudaMemcpyAsync(&lp, base, 8, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "exchange");
    return lp;
}

void Engine::swap(uint64_t left, uint64_t right) {
    if (left >= walkers_ || right >= walkers_) throw WlgError(WLG_ERR_OUT_OF_RANGE, "walker index out of range");
    char* base = d_scratch_.get<char>();
    launch_exchange_pair(view_, static_cast<int>(left), static_cast<int>(right), 1, reinterpret_cast<double*>(base),
                         reinterpret_cast<int*>(base + 16), stream_);
    int status = 0;
    check_cuda(cudaMemcpyAsync(&status, base + 16, sizeof status, cudaMemcpyDeviceToHost, stream_), "copy");
    check_cuda(cudaStreamSynchronize(stream_), "swap");
    if (status) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Replica exchange would violate an energy window");
}

// Warm start (no counterpart in the reference, whose walkers start from log g = 0 and
// ln f = 1): before the first attempt, every walker's window slice of log g is set from a
// whole-grid estimate and its refinement factor to `factor`.  Bins outside the windows stay
// zero, as in a fresh walker.
void Engine::warm_start(const double* log_g, double factor, bool continue_schedule) {
    if (!log_g) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "null log g estimate");
    if (!std::isfinite(factor) || !(factor > 0.0))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "The warm-start factor must be finite and positive");
    std::vector<WalkerState> states = download_states();
    for (const WalkerState& st : states)
        if (st.attempted != 0) throw WlgError(WLG_ERR_LOGIC, "A warm start must precede the first attempt");
    for (uint64_t w = 0; w < windows_; ++w)
        for (uint64_t b = win_[2 * w]; b < win_[2 * w + 1]; ++b)
            if (!std::isfinite(log_g[b]))
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "The log g estimate must be finite inside every window");
    std::vector<double> grid(walkers_ * bins_, 0.0);
    for (uint64_t k = 0; k < walkers_; ++k) {
        const WalkerState& st = states[k];
        for (uint64_t b = win_[2 * st.window]; b < win_[2 * st.window + 1]; ++b) grid[k * bins_ + b] = log_g[b];
        states[k].factor = factor;
        states[k].stage = factor <= p_.final_factor ? kFrozen : kWangLandau;
        // continuing the 1/t schedule: the offset is set at the first covered check
        states[k].time_offset = continue_schedule ? kContinueSchedule : 0;
    }
    check_cuda(cudaMemcpyAsync(d_log_g_.ptr, grid.data(), grid.size() * sizeof(double), cudaMemcpyHostToDevice,
                               stream_),
               "copy log g");
    check_cuda(cudaMemcpyAsync(d_ws_.ptr, states.data(), states.size() * sizeof(WalkerState), cudaMemcpyHostToDevice,
                               stream_),
               "copy states");
    check_cuda(cudaStreamSynchronize(stream_), "sync");
}

// ---- multi-walker run checkpoint -------------------------------------------------------
//
// Binary layout (host byte order): RunHeader, window bounds (2 x windows uint64), Control,
// PrecisionReport, then per walker in walker order WalkerState and the walker's spins (ld
// bytes) and fields (ld doubles), then the whole-grid estimator arrays (W x bins: log g,
// H, active; with pilot statistics or the Nalivaiko mask also the refinement mask, the
// squared displacements and their sample counts; with pilot statistics the representative
// bank).  A restore puts walker w's configuration in slot w.

namespace {
struct RunHeader {
    char magic[8];
    uint64_t walkers, windows, n, ld, bins, seed, system_hash;
    int32_t precision, features, collect, pad;
    double emin, emax, width;
    uint64_t recomputes, next_recompute_in;  // epochs until the next FP64 recompute
};
constexpr char kRunMagic[8] = {'W', 'L', 'G', 'R', 'U', 'N', '0', '1'};

template <class T> void put_raw(std::ofstream& out, const T* p, size_t count) {
    out.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(count * sizeof(T)));
}
template <class T> void get_raw(std::ifstream& in, T* p, size_t count) {
    in.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(count * sizeof(T)));
    if (!in) throw WlgError(WLG_ERR_IO, "Run checkpoint is truncated");
}
template <class T> std::vector<T> download(const DeviceBuffer& b, size_t count, cudaStream_t s) {
    std::vector<T> v(count);
    if (count) check_cuda(cudaMemcpyAsync(v.data(), b.ptr, count * sizeof(T), cudaMemcpyDeviceToHost, s), "copy");
    return v;
}
template <class T> void upload(DeviceBuffer& b, const std::vector<T>& v, cudaStream_t s) {
    if (!v.empty())
        check_cuda(cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "copy");
}
}  // namespace

void Engine::save_run(const std::string& path) {
    const size_t W = walkers_, B = bins_, ld = sys_.ld, WB = W * B;
    const size_t R = p_.collect ? W * kRepresentatives : 0;
    Control ctl{};
    PrecisionReport rep{};
    check_cuda(cudaMemcpyAsync(&ctl, d_ctl_.ptr, sizeof ctl, cudaMemcpyDeviceToHost, stream_), "copy control");
    check_cuda(cudaMemcpyAsync(&rep, d_prec_.ptr, sizeof rep, cudaMemcpyDeviceToHost, stream_), "copy report");
    std::vector<WalkerState> st = download<WalkerState>(d_ws_, W, stream_);
    std::vector<int8_t> spins = download<int8_t>(d_spins_, W * ld, stream_);
    std::vector<double> fields = download<double>(d_fields_, W * ld, stream_);
    std::vector<double> lg = download<double>(d_log_g_, WB, stream_);
    std::vector<uint64_t> h = download<uint64_t>(d_hist_, WB, stream_);
    std::vector<uint8_t> act = download<uint8_t>(d_active_, WB, stream_);
    std::vector<uint8_t> ref = download<uint8_t>(d_refine_, features_ ? WB : 0, stream_);
    std::vector<double> sq = download<double>(d_sqdisp_, features_ ? WB : 0, stream_);
    std::vector<uint64_t> ds = download<uint64_t>(d_dsamples_, features_ ? WB : 0, stream_);
    std::vector<double> re = download<double>(d_rep_energy_, R, stream_), rd = download<double>(d_rep_dist_, R, stream_),
                        rt = download<double>(d_rep_target_, R, stream_);
    std::vector<uint8_t> rp = download<uint8_t>(d_rep_present_, R, stream_);
    std::vector<int8_t> rs = download<int8_t>(d_rep_spins_, R * ld, stream_);
    check_cuda(cudaStreamSynchronize(stream_), "checkpoint");

    RunHeader hd{};
    std::memcpy(hd.magic, kRunMagic, 8);
    hd.walkers = W;
    hd.windows = windows_;
    hd.n = sys_.n;
    hd.ld = ld;
    hd.bins = B;
    hd.seed = p_.seed;
    hd.system_hash = system_hash_;
    hd.precision = precision_;
    hd.features = features_ ? 1 : 0;
    hd.collect = p_.collect ? 1 : 0;
    hd.emin = cfg_.emin;
    hd.emax = cfg_.emax;
    hd.width = cfg_.bin_width;
    hd.recomputes = rep.recomputes;
    hd.next_recompute_in = next_recompute_ > epochs_ ? next_recompute_ - epochs_ : 0;
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::binary | std::ios::trunc);
        if (!out) throw WlgError(WLG_ERR_IO, "Cannot write run checkpoint " + tmp);
        put_raw(out, &hd, 1);
        put_raw(out, win_.data(), win_.size());
        put_raw(out, &ctl, 1);
        put_raw(out, &rep, 1);
        for (size_t w = 0; w < W; ++w) {
            put_raw(out, &st[w], 1);
            put_raw(out, spins.data() + static_cast<size_t>(st[w].slot) * ld, ld);
            put_raw(out, fields.data() + static_cast<size_t>(st[w].slot) * ld, ld);
        }
        put_raw(out, lg.data(), WB);
        put_raw(out, h.data(), WB);
        put_raw(out, act.data(), WB);
        if (features_) {
            put_raw(out, ref.data(), WB);
            put_raw(out, sq.data(), WB);
            put_raw(out, ds.data(), WB);
        }
        if (R) {
            put_raw(out, re.data(), R);
            put_raw(out, rd.data(), R);
            put_raw(out, rt.data(), R);
            put_raw(out, rp.data(), R);
            put_raw(out, rs.data(), R * ld);
        }
        out.flush();
        if (!out) throw WlgError(WLG_ERR_IO, "Cannot write run checkpoint " + tmp);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw WlgError(WLG_ERR_IO, "Cannot replace " + path);
}

void Engine::load_run(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw WlgError(WLG_ERR_IO, "Cannot open run checkpoint " + path);
    const size_t W = walkers_, B = bins_, ld = sys_.ld, WB = W * B;
    const size_t R = p_.collect ? W * kRepresentatives : 0;
    RunHeader hd{};
    get_raw(in, &hd, 1);
    if (std::memcmp(hd.magic, kRunMagic, 8) != 0) throw WlgError(WLG_ERR_IO, "Not a run checkpoint");
    if (hd.walkers != W || hd.windows != windows_ || hd.n != sys_.n || hd.ld != ld || hd.bins != B ||
        hd.system_hash != system_hash_ || hd.precision != precision_ || hd.features != (features_ ? 1 : 0) ||
        hd.collect != (p_.collect ? 1 : 0) || hd.emin != cfg_.emin || hd.emax != cfg_.emax ||
        hd.width != cfg_.bin_width)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Run checkpoint is incompatible with this run");
    std::vector<uint64_t> win(win_.size());
    get_raw(in, win.data(), win.size());
    if (win != win_) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Run checkpoint has other energy windows");
    Control ctl{};
    PrecisionReport rep{};
    get_raw(in, &ctl, 1);
    get_raw(in, &rep, 1);
    std::vector<WalkerState> st(W);
    std::vector<int8_t> spins(W * ld);
    std::vector<double> fields(W * ld);
    for (size_t w = 0; w < W; ++w) {
        get_raw(in, &st[w], 1);
        get_raw(in, spins.data() + w * ld, ld);
        get_raw(in, fields.data() + w * ld, ld);
        st[w].slot = static_cast<int32_t>(w);
        if (st[w].window != static_cast<int32_t>(w / wpw_))
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Run checkpoint walker order mismatch");
    }
    std::vector<double> lg(WB);
    std::vector<uint64_t> h(WB);
    std::vector<uint8_t> act(WB);
    get_raw(in, lg.data(), WB);
    get_raw(in, h.data(), WB);
    get_raw(in, act.data(), WB);
    std::vector<uint8_t> ref;
    std::vector<double> sq;
    std::vector<uint64_t> ds;
    if (features_) {
        ref.resize(WB);
        sq.resize(WB);
        ds.resize(WB);
        get_raw(in, ref.data(), WB);
        get_raw(in, sq.data(), WB);
        get_raw(in, ds.data(), WB);
    }
    std::vector<double> re(R), rd(R), rt(R);
    std::vector<uint8_t> rp(R);
    std::vector<int8_t> rs(R * ld);
    if (R) {
        get_raw(in, re.data(), R);
        get_raw(in, rd.data(), R);
        get_raw(in, rt.data(), R);
        get_raw(in, rp.data(), R);
        get_raw(in, rs.data(), R * ld);
    }
    check_cuda(cudaMemcpyAsync(d_ctl_.ptr, &ctl, sizeof ctl, cudaMemcpyHostToDevice, stream_), "copy control");
    check_cuda(cudaMemcpyAsync(d_prec_.ptr, &rep, sizeof rep, cudaMemcpyHostToDevice, stream_), "copy report");
    upload(d_ws_, st, stream_);
    upload(d_spins_, spins, stream_);
    upload(d_fields_, fields, stream_);
    upload(d_log_g_, lg, stream_);
    upload(d_hist_, h, stream_);
    upload(d_active_, act, stream_);
    if (features_) {
        upload(d_refine_, ref, stream_);
        upload(d_sqdisp_, sq, stream_);
        upload(d_dsamples_, ds, stream_);
    }
    if (R) {
        upload(d_rep_energy_, re, stream_);
        upload(d_rep_dist_, rd, stream_);
        upload(d_rep_target_, rt, stream_);
        upload(d_rep_present_, rp, stream_);
        upload(d_rep_spins_, rs, stream_);
    }
    check_cuda(cudaStreamSynchronize(stream_), "restore");
    done_ = ctl.done != 0;
    epochs_ = ctl.epoch;
    if (recompute_epochs_) next_recompute_ = epochs_ + hd.next_recompute_in;
    last_checkpoint_ = st[0].attempted;
}

}  // namespace wlg
