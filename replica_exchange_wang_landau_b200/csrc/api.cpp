// api.cpp — the extern "C" boundary declared in include/wlg.h.  Exceptions never cross it:
// every entry point returns a wlg_status and records the message for wlg_last_error().
#include <cmath>
#include <limits>
#include <new>

#include "engine.hpp"

struct wlg_engine {
    wlg::Engine* impl;
};

namespace {

thread_local std::string g_last_error;

wlg_status fail(wlg_status s, const std::string& message) {
    g_last_error = message;
    return s;
}

template <class F> wlg_status guarded(F&& f) {
    try {
        g_last_error.clear();
        f();
        return WLG_OK;
    } catch (const wlg::WlgError& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(WLG_ERR_RUNTIME, "out of host memory");
    } catch (const std::exception& e) {
        return fail(WLG_ERR_RUNTIME, e.what());
    }
}

// attempts_from_mcs (src/io.cpp:75-87)
uint64_t attempts_from_mcs(double mcs, uint64_t n, bool allow_zero) {
    if (n == 0) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "Cannot resolve MCS for an empty system");
    if (!std::isfinite(mcs) || mcs < 0.0 || (!allow_zero && mcs == 0.0))
        throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid MCS value");
    if (mcs == 0.0) return 0;
    const long double raw = static_cast<long double>(mcs) * static_cast<long double>(n);
    const auto rounded = static_cast<uint64_t>(std::floor(raw + 0.5L));
    return std::max<uint64_t>(1, rounded);
}

// A stand-alone device system with its couplings, for the physics entry points.
struct Standalone {
    cudaStream_t stream = nullptr;
    wlg::DeviceSystem sys;
    wlg::EngineView view{};
    Standalone(const wlg_system& s, int precision) {
        wlg::validate_system(s);
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
            throw wlg::WlgError(WLG_ERR_DEVICE, "No CUDA device is available; this library runs on an sm_100 GPU only");
        wlg::check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        wlg::upload_system(s, sys, stream);
        wlg::build_couplings(sys, precision, stream);
        view.n = static_cast<int32_t>(sys.n);
        view.ld = static_cast<int32_t>(sys.ld);
        view.csr = sys.csr ? 1 : 0;
        view.precision = precision;
        view.J64 = sys.J64.get<double>();
        view.csr_ptr = sys.csr_ptr.get<int32_t>();
        view.csr_col = sys.csr_col.get<int32_t>();
        view.csr_val64 = sys.csr_val64.get<double>();
    }
    ~Standalone() {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

float bf16_to_float(uint16_t b) {
    const uint32_t w = static_cast<uint32_t>(b) << 16;
    float f;
    std::memcpy(&f, &w, 4);
    return f;
}

}  // namespace

extern "C" {

int32_t wlg_abi_version(void) { return WLG_ABI_VERSION; }

const char* wlg_last_error(void) { return g_last_error.c_str(); }

wlg_status wlg_set_device(int32_t device) {
    return guarded([&] { wlg::check_cuda(cudaSetDevice(device), "cudaSetDevice"); });
}

wlg_status wlg_default_run_config(uint64_t n, wlg_run_config* out) {
    return guarded([&] {
        if (!out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        wlg_run_config c{};
        c.emin = -20.0;
        c.emax = 20.0;
        c.bin_width = 0.1;
        c.windows = 1;
        c.walkers_per_window = 1;
        c.overlap = 0.75;
        c.seed = 1;
        c.wl.flatness = 0.8;
        c.wl.minimum_visits = 100;
        c.wl.final_factor = 1e-8;
        c.wl.check_interval_attempts = attempts_from_mcs(100.0, n, false);
        c.wl.force_accept_after_attempts = attempts_from_mcs(0.0, n, true);
        c.wl.inverse_time_enabled = 1;
        c.wl.initialization_max_attempts = 1'000'000;
        c.wl.initialization_target_fraction = 0.5;
        c.wl.initialization_temperature_fraction = 0.05;
        c.wl.initialization_stall_attempts_per_spin = 1'000;
        c.wl.initialization_temperature_multiplier = 2.0;
        c.wl.initialization_max_temperature_fraction = 0.5;
        c.wl.collect_window_statistics = 0;
        c.wl.round_trip_margin_fraction = 0.1;
        c.wl.nalivaiko_mod = 0;
        c.exchange_interval_attempts = attempts_from_mcs(10.0, n, false);
        c.max_attempts = attempts_from_mcs(1'000'000.0, n, true);
        c.checkpoint_interval_attempts = attempts_from_mcs(10'000.0, n, false);
        c.coupling_precision = WLG_PRECISION_FP64;
        c.recompute_interval_attempts = n;
        *out = c;
    });
}

wlg_status wlg_grid_bins(double emin, double emax, double width, uint64_t* bins) {
    return guarded([&] { *bins = wlg::grid_bins(emin, emax, width); });
}

wlg_status wlg_grid_index(double emin, double emax, double width, double energy, int64_t* bin) {
    return guarded([&] {
        const uint64_t count = wlg::grid_bins(emin, emax, width);
        *bin = wlg::grid_index(wlg::make_grid(emin, emax, width, static_cast<int64_t>(count)), energy);
    });
}

wlg_status wlg_partition_windows(uint64_t bins, uint64_t count, double overlap, uint64_t* out) {
    return guarded([&] {
        const auto w = wlg::partition_windows(bins, count, overlap);
        std::copy(w.begin(), w.end(), out);
    });
}

wlg_status wlg_validate_system(const wlg_system* system) {
    return guarded([&] {
        if (!system) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null system");
        wlg::validate_system(*system);
    });
}

wlg_status wlg_checkpoint_save(const char* path, const wlg_snapshot* s, uint64_t n_spins, uint64_t n_bins) {
    return guarded([&] {
        if (!path || !s) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::save_checkpoint_file(path, *s, n_spins, n_bins);
    });
}

wlg_status wlg_checkpoint_load(const char* path, wlg_snapshot* s, uint64_t* n_spins, uint64_t* n_bins) {
    return guarded([&] {
        if (!path || !s || !n_spins || !n_bins) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        std::vector<int8_t> sp;
        std::vector<double> fl, lg;
        std::vector<uint64_t> hs;
        std::vector<uint8_t> ac;
        wlg_snapshot scalars{};
        std::string error;
        if (!wlg::load_checkpoint_file(path, sp, fl, lg, hs, ac, scalars, error))
            throw wlg::WlgError(error.rfind("Cannot open", 0) == 0 ? WLG_ERR_IO : WLG_ERR_RUNTIME, error);
        if (fl.size() != sp.size() || hs.size() != lg.size() || ac.size() != lg.size())
            throw wlg::WlgError(WLG_ERR_RUNTIME, "Checkpoint vectors have inconsistent sizes");
        const bool sizes_only = !s->spins || !s->fields || !s->log_g || !s->histogram || !s->active;
        if (!sizes_only && (*n_spins < sp.size() || *n_bins < lg.size()))
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "checkpoint buffers too small");
        *n_spins = sp.size();
        *n_bins = lg.size();
        if (sizes_only) return;
        std::memcpy(s->spins, sp.data(), sp.size());
        std::memcpy(s->fields, fl.data(), fl.size() * 8);
        std::memcpy(s->log_g, lg.data(), lg.size() * 8);
        std::memcpy(s->histogram, hs.data(), hs.size() * 8);
        std::memcpy(s->active, ac.data(), ac.size());
        s->walker_id = scalars.walker_id;
        s->energy = scalars.energy;
        s->factor = scalars.factor;
        s->attempted = scalars.attempted;
        s->accepted = scalars.accepted;
        s->forced_accepted = scalars.forced_accepted;
        s->last_accepted_attempt = scalars.last_accepted_attempt;
        s->stage = scalars.stage;
        for (int k = 0; k < 4; ++k) s->rng_state[k] = scalars.rng_state[k];
    });
}

wlg_status wlg_couplings_dense(const wlg_system* system, int32_t precision, double* out) {
    return guarded([&] {
        if (!system || !out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        if (precision < WLG_PRECISION_FP64 || precision > WLG_PRECISION_BF16 ||
            (system->cutoff > 0.0 && precision == WLG_PRECISION_BF16))
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "Unsupported coupling precision");
        Standalone s(*system, precision);
        const uint64_t n = s.sys.n, ld = s.sys.ld;
        std::fill(out, out + n * n, 0.0);
        if (!s.sys.csr) {
            if (precision == WLG_PRECISION_FP64) {
                std::vector<double> J(ld * ld);
                wlg::check_cuda(cudaMemcpyAsync(J.data(), s.sys.J64.ptr, ld * ld * 8, cudaMemcpyDeviceToHost, s.stream), "copy");
                wlg::check_cuda(cudaStreamSynchronize(s.stream), "sync");
                for (uint64_t i = 0; i < n; ++i) std::memcpy(out + i * n, J.data() + i * ld, n * 8);
            } else if (precision == WLG_PRECISION_FP32) {
                std::vector<float> J(ld * ld);
                wlg::check_cuda(cudaMemcpyAsync(J.data(), s.sys.J32.ptr, ld * ld * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
                wlg::check_cuda(cudaStreamSynchronize(s.stream), "sync");
                for (uint64_t i = 0; i < n; ++i)
                    for (uint64_t j = 0; j < n; ++j) out[i * n + j] = static_cast<double>(J[i * ld + j]);
            } else {
                std::vector<uint16_t> J(ld * ld);
                std::vector<float> scale(ld);
                wlg::check_cuda(cudaMemcpyAsync(J.data(), s.sys.J16.ptr, ld * ld * 2, cudaMemcpyDeviceToHost, s.stream), "copy");
                wlg::check_cuda(cudaMemcpyAsync(scale.data(), s.sys.Jscale.ptr, ld * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
                wlg::check_cuda(cudaStreamSynchronize(s.stream), "sync");
                for (uint64_t i = 0; i < n; ++i)
                    for (uint64_t j = 0; j < n; ++j)
                        out[i * n + j] = static_cast<double>(bf16_to_float(J[i * ld + j])) * static_cast<double>(scale[i]);
            }
            return;
        }
        std::vector<int32_t> ptr(n + 1), col(std::max<uint64_t>(1, s.sys.nnz));
        std::vector<double> v64(std::max<uint64_t>(1, s.sys.nnz));
        std::vector<float> v32(std::max<uint64_t>(1, s.sys.nnz));
        wlg::check_cuda(cudaMemcpyAsync(ptr.data(), s.sys.csr_ptr.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaMemcpyAsync(col.data(), s.sys.csr_col.ptr, s.sys.nnz * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaMemcpyAsync(v64.data(), s.sys.csr_val64.ptr, s.sys.nnz * 8, cudaMemcpyDeviceToHost, s.stream), "copy");
        if (precision == WLG_PRECISION_FP32)
            wlg::check_cuda(cudaMemcpyAsync(v32.data(), s.sys.csr_val32.ptr, s.sys.nnz * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaStreamSynchronize(s.stream), "sync");
        for (uint64_t i = 0; i < n; ++i)
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                out[i * n + static_cast<uint64_t>(col[k])] =
                    precision == WLG_PRECISION_FP32 ? static_cast<double>(v32[k]) : v64[k];
    });
}

wlg_status wlg_couplings_csr(const wlg_system* system, uint64_t* nnz, uint64_t* row_offsets, uint64_t* columns,
                             double* values) {
    return guarded([&] {
        if (!system || !nnz) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        if (!(system->cutoff > 0.0)) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR cutoff must be positive");
        Standalone s(*system, WLG_PRECISION_FP64);
        const uint64_t n = s.sys.n;
        *nnz = s.sys.nnz;
        if (!columns) return;
        std::vector<int32_t> ptr(n + 1), col(std::max<uint64_t>(1, s.sys.nnz));
        wlg::check_cuda(cudaMemcpyAsync(ptr.data(), s.sys.csr_ptr.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaMemcpyAsync(col.data(), s.sys.csr_col.ptr, s.sys.nnz * 4, cudaMemcpyDeviceToHost, s.stream), "copy");
        if (values)
            wlg::check_cuda(cudaMemcpyAsync(values, s.sys.csr_val64.ptr, s.sys.nnz * 8, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaStreamSynchronize(s.stream), "sync");
        if (row_offsets)
            for (uint64_t i = 0; i <= n; ++i) row_offsets[i] = static_cast<uint64_t>(ptr[i]);
        for (uint64_t k = 0; k < s.sys.nnz; ++k) columns[k] = static_cast<uint64_t>(col[k]);
    });
}

wlg_status wlg_local_fields(const wlg_system* system, const int8_t* spins, uint64_t count, double* fields,
                            double* energies) {
    return guarded([&] {
        if (!system || !spins || !fields) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        for (uint64_t k = 0; k < count * system->n; ++k)
            if (spins[k] != 1 && spins[k] != -1) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "Spins must be +/-1");
        if (count == 0) return;
        Standalone s(*system, WLG_PRECISION_FP64);
        const uint64_t n = s.sys.n;
        wlg::DeviceBuffer d_s(count * n), d_f(count * n * 8), d_e(count * 8);
        wlg::check_cuda(cudaMemcpyAsync(d_s.ptr, spins, count * n, cudaMemcpyHostToDevice, s.stream), "copy");
        wlg::compute_fields(s.view, d_s.get<int8_t>(), static_cast<int64_t>(n), d_f.get<double>(),
                            static_cast<int64_t>(n), d_e.get<double>(), static_cast<int>(count), s.stream);
        wlg::check_cuda(cudaMemcpyAsync(fields, d_f.ptr, count * n * 8, cudaMemcpyDeviceToHost, s.stream), "copy");
        if (energies)
            wlg::check_cuda(cudaMemcpyAsync(energies, d_e.ptr, count * 8, cudaMemcpyDeviceToHost, s.stream), "copy");
        wlg::check_cuda(cudaStreamSynchronize(s.stream), "local_fields");
    });
}

wlg_status wlg_local_fields_noalloc(const wlg_system* system, const int8_t* spins, uint64_t count, double* fields,
                                    double* energies) {
    return guarded([&] {
        if (!system || !spins || !fields) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::local_fields_noalloc(*system, spins, count, fields, energies);
    });
}

wlg_status wlg_engine_create(const wlg_system* system, const wlg_run_config* config, wlg_engine** engine) {
    return guarded([&] {
        if (!system || !config || !engine) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        *engine = nullptr;
        auto* impl = new wlg::Engine(*system, *config);
        *engine = new wlg_engine{impl};
    });
}

wlg_status wlg_engine_create_from_couplings(const wlg_couplings* couplings, const wlg_run_config* config,
                                            wlg_engine** engine) {
    return guarded([&] {
        if (!couplings || !config || !engine) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        *engine = nullptr;
        auto* impl = new wlg::Engine(*couplings, *config);
        *engine = new wlg_engine{impl};
    });
}

void wlg_engine_destroy(wlg_engine* engine) {
    if (!engine) return;
    if (engine->impl) cudaSetDevice(engine->impl->device);
    delete engine->impl;
    delete engine;
}

#define WLG_ENGINE_GUARD(engine)                                                                 \
    if (!(engine) || !(engine)->impl) return fail(WLG_ERR_INVALID_ARGUMENT, "null engine");  \
    if (cudaSetDevice((engine)->impl->device) != cudaSuccess)                                    \
        return fail(WLG_ERR_DEVICE, "cannot select the engine's CUDA device");

wlg_status wlg_engine_stitch(wlg_engine* engine, int32_t complete_range, double* log_g, uint64_t* histogram,
                             double* standard_error, uint8_t* valid, wlg_join_quality* joins,
                             int32_t* fully_normalized) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!log_g || !histogram || !standard_error || !valid)
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output array");
        engine->impl->stitch(complete_range, log_g, histogram, standard_error, valid, joins, fully_normalized);
    });
}

wlg_status wlg_engine_set_staging_ring(wlg_engine* engine, int32_t entries) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->set_staging_ring(entries); });
}

wlg_status wlg_engine_inject_wait_timeout(wlg_engine* engine) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->inject_wait_timeout(); });
}

wlg_status wlg_engine_run(wlg_engine* engine, wlg_run_totals* totals) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->run(totals); });
}

wlg_status wlg_engine_run_epochs(wlg_engine* engine, uint64_t max_epochs, uint64_t* epochs_run, int32_t* done) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->run_epochs(max_epochs, epochs_run, done); });
}

wlg_status wlg_engine_totals(wlg_engine* engine, wlg_run_totals* totals) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->totals(totals); });
}

wlg_status wlg_engine_time_epochs(wlg_engine* engine, uint64_t epochs, wlg_epoch_timing* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        engine->impl->time_epochs(epochs, out);
    });
}

wlg_status wlg_engine_time_run(wlg_engine* engine, uint64_t epochs, wlg_epoch_timing* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        engine->impl->time_run(epochs, out);
    });
}

wlg_status wlg_engine_save_run(wlg_engine* engine, const char* path) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!path || !path[0]) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "empty checkpoint path");
        engine->impl->save_run(path);
    });
}

wlg_status wlg_engine_load_run(wlg_engine* engine, const char* path) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!path || !path[0]) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "empty checkpoint path");
        engine->impl->load_run(path);
    });
}

wlg_status wlg_engine_autotune(wlg_engine* engine, uint64_t trial_epochs, wlg_autotune_report* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->autotune(trial_epochs, out); });
}

wlg_status wlg_engine_precision_report(wlg_engine* engine, wlg_precision_report* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        engine->impl->precision_report(out);
    });
}

wlg_status wlg_engine_warm_start(wlg_engine* engine, const double* log_g, double factor) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->warm_start(log_g, factor); });
}

wlg_status wlg_engine_warm_start_continue(wlg_engine* engine, const double* log_g, double factor) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->warm_start(log_g, factor, true); });
}

wlg_status wlg_engine_set_launch(wlg_engine* engine, int32_t walkers_per_block, int32_t epochs_per_graph) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->set_launch(walkers_per_block, epochs_per_graph); });
}

wlg_status wlg_engine_set_window_sweep(wlg_engine* engine, int32_t enabled) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->set_window_sweep(enabled != 0); });
}

int32_t wlg_engine_window_sweep(const wlg_engine* engine) {
    return engine && engine->impl && engine->impl->window_sweep() ? 1 : 0;
}

uint64_t wlg_engine_walkers(const wlg_engine* engine) { return engine && engine->impl ? engine->impl->walkers() : 0; }
uint64_t wlg_engine_bins(const wlg_engine* engine) { return engine && engine->impl ? engine->impl->bins() : 0; }
uint64_t wlg_engine_spins(const wlg_engine* engine) { return engine && engine->impl ? engine->impl->spins() : 0; }

wlg_status wlg_engine_window(const wlg_engine* engine, uint64_t w, uint64_t* begin, uint64_t* end) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->window(w, begin, end); });
}

wlg_status wlg_engine_fragment(wlg_engine* engine, uint64_t w, int32_t allow_empty, double* log_g,
                               uint64_t* histogram, double* standard_error, uint8_t* valid) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->fragment(w, allow_empty, log_g, histogram, standard_error, valid); });
}

wlg_status wlg_engine_fragments(wlg_engine* engine, int32_t allow_empty, double* log_g, uint64_t* histogram,
                                double* standard_error, uint8_t* valid) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        if (!log_g || !histogram || !standard_error || !valid)
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        engine->impl->fragments(allow_empty, log_g, histogram, standard_error, valid);
    });
}

wlg_status wlg_engine_sampling_statistics(wlg_engine* engine, uint64_t w, double* squared_energy_displacement,
                                          uint64_t* displacement_samples, uint64_t* round_trips, uint64_t* walkers) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        engine->impl->sampling(w, squared_energy_displacement, displacement_samples, round_trips, walkers);
    });
}

wlg_status wlg_engine_walker_statistics(wlg_engine* engine, wlg_walker_statistics* out, uint64_t capacity) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->walker_statistics(out, capacity); });
}

wlg_status wlg_engine_representatives(wlg_engine* engine, double* energies, int8_t* spins, uint64_t capacity,
                                      uint64_t* count) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->representatives(energies, spins, capacity, count); });
}

wlg_status wlg_walker_run_attempts(wlg_engine* engine, uint64_t walker, uint64_t count) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->run_attempts(walker, count); });
}

wlg_status wlg_walker_snapshot(wlg_engine* engine, uint64_t walker, wlg_snapshot* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->snapshot(walker, out); });
}

wlg_status wlg_walker_restore(wlg_engine* engine, uint64_t walker, const wlg_snapshot* in) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->restore(walker, *in); });
}

wlg_status wlg_walker_histogram_statistics(wlg_engine* engine, uint64_t walker, wlg_histogram_statistics* out) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->histogram_statistics(walker, out, nullptr); });
}

wlg_status wlg_walker_flags(wlg_engine* engine, uint64_t walker, int32_t* flat, int32_t* covered, int32_t* ready) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] {
        wlg_histogram_statistics s{};
        int32_t f[3];
        engine->impl->histogram_statistics(walker, &s, f);
        if (flat) *flat = f[0];
        if (covered) *covered = f[1];
        if (ready) *ready = f[2];
    });
}

wlg_status wlg_walker_begin_next_iteration(wlg_engine* engine, uint64_t walker) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->begin_next_iteration(walker); });
}

wlg_status wlg_walker_exchange_log_probability(wlg_engine* engine, uint64_t left, uint64_t right,
                                               double* log_probability) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { *log_probability = engine->impl->exchange_log_probability(left, right); });
}

wlg_status wlg_walker_swap(wlg_engine* engine, uint64_t left, uint64_t right) {
    WLG_ENGINE_GUARD(engine)
    return guarded([&] { engine->impl->swap(left, right); });
}

}  // extern "C"

// ---- the warm-start network (no counterpart in the reference) ----------------------------

extern "C" {

struct wlg_mlp {
    wlg::Mlp* impl;
};

wlg_status wlg_mlp_create(int32_t layers, const int32_t* dims, uint64_t seed, wlg_mlp** out) {
    return guarded([&] {
        if (!dims || !out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        wlg::Mlp* m = wlg::mlp_create(layers, dims, seed);
        *out = new wlg_mlp{m};
    });
}

void wlg_mlp_destroy(wlg_mlp* mlp) {
    if (!mlp) return;
    wlg::mlp_destroy(mlp->impl);
    delete mlp;
}

uint64_t wlg_mlp_parameter_count(const wlg_mlp* mlp) { return mlp ? wlg::mlp_count(mlp->impl) : 0; }

wlg_status wlg_mlp_get_parameters(wlg_mlp* mlp, float* out) {
    return guarded([&] {
        if (!mlp || !out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::mlp_get(mlp->impl, out);
    });
}

wlg_status wlg_mlp_set_parameters(wlg_mlp* mlp, const float* in) {
    return guarded([&] {
        if (!mlp || !in) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::mlp_set(mlp->impl, in);
    });
}

wlg_status wlg_mlp_forward(wlg_mlp* mlp, const float* x, uint64_t batch, float* y) {
    return guarded([&] {
        if (!mlp || !x || !y) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::mlp_forward(mlp->impl, x, batch, y);
    });
}

wlg_status wlg_mlp_gradients(wlg_mlp* mlp, const float* x, const float* t, uint64_t batch, float* grads,
                             double* loss) {
    return guarded([&] {
        if (!mlp || !x || !t || !grads || !loss) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        *loss = wlg::mlp_gradients(mlp->impl, x, t, batch, grads);
    });
}

wlg_status wlg_mlp_train(wlg_mlp* mlp, const float* x, const float* t, uint64_t batch, uint64_t steps,
                         double learning_rate, double* loss) {
    return guarded([&] {
        if (!mlp || !x || !t || !loss) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        if (!(learning_rate > 0.0) || !std::isfinite(learning_rate))
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "learning rate must be positive");
        *loss = wlg::mlp_train(mlp->impl, x, t, batch, steps, learning_rate);
    });
}

// ---- batches of engines (no counterpart in the reference) ---------------------------------

struct wlg_batch {
    wlg::Batch* impl;
};

wlg_status wlg_batch_create(wlg_engine* const* engines, uint64_t count, wlg_batch** out) {
    return guarded([&] {
        if (!engines || !out || count == 0) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        std::vector<wlg::Engine*> list;
        for (uint64_t k = 0; k < count; ++k) {
            if (!engines[k]) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null engine in a batch");
            list.push_back(engines[k]->impl);
        }
        wlg::check_cuda(cudaSetDevice(list[0]->device), "cudaSetDevice");
        *out = new wlg_batch{new wlg::Batch(list)};
    });
}

wlg_status wlg_batch_run_epochs(wlg_batch* batch, uint64_t max_epochs, uint64_t* launches, int32_t* all_done) {
    return guarded([&] {
        if (!batch) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null batch");
        batch->impl->run_epochs(max_epochs, launches, all_done);
    });
}

void wlg_batch_destroy(wlg_batch* batch) {
    if (!batch) return;
    delete batch->impl;
    delete batch;
}

// ---- stitching and output -------------------------------------------------------------

wlg_status wlg_stitch_dos(double emin, double emax, double width, const wlg_fragment_view* fragments,
                          uint64_t count, int32_t complete_range, uint64_t spin_count, double* log_g,
                          uint64_t* histogram, double* standard_error, uint8_t* valid, wlg_join_quality* joins,
                          int32_t* fully_normalized) {
    return guarded([&] {
        if (!log_g || !histogram || !standard_error || !valid)
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null output");
        wlg::stitch_dos(emin, emax, width, fragments, count, complete_range != 0, spin_count, log_g, histogram,
                        standard_error, valid, joins, fully_normalized);
    });
}

wlg_status wlg_write_dos_csv(const char* path, double emin, double width, uint64_t bins, const double* log_g,
                             const uint64_t* histogram, const double* standard_error, const uint8_t* valid) {
    return guarded([&] {
        if (!path || !log_g || !histogram || !standard_error || !valid)
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::write_dos_csv(path, emin, width, bins, log_g, histogram, standard_error, valid);
    });
}

wlg_status wlg_write_fragment_csv(const char* path, double emin, double width, uint64_t window_id,
                                  uint64_t window_begin, uint64_t window_end, const double* log_g,
                                  const uint64_t* histogram, const double* standard_error, const uint8_t* valid) {
    return guarded([&] {
        if (!path || !log_g || !histogram || !standard_error || !valid)
            throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::write_fragment_csv(path, emin, width, window_id, window_begin, window_end, log_g, histogram,
                                standard_error, valid);
    });
}

wlg_status wlg_write_workers_stat_csv(const char* path, const wlg_walker_statistics* statistics, uint64_t count,
                                      uint64_t spin_count) {
    return guarded([&] {
        if (!path || (count != 0 && !statistics)) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::write_workers_stat_csv(path, statistics, count, spin_count);
    });
}

// ---- the adaptive-window pilot's host steps ------------------------------------------

wlg_status wlg_adapt_energy_windows(double emin, double emax, double width, const wlg_fragment_view* fragments,
                                    const wlg_sampling_view* sampling, uint64_t count, double overlap,
                                    const wlg_adaptive_parameters* parameters, uint64_t* windows_out) {
    return guarded([&] {
        if (!parameters || !windows_out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        const auto w = wlg::adapt_energy_windows(emin, emax, width, fragments, sampling, count, overlap, *parameters);
        std::copy(w.begin(), w.end(), windows_out);
    });
}

wlg_status wlg_select_initial_configurations(double emin, double emax, double width, const uint64_t* windows,
                                             uint64_t count, const double* representative_energy,
                                             const int8_t* representative_spins, const uint8_t* representative_present,
                                             uint64_t representatives, uint64_t spins, uint64_t walkers_per_window,
                                             int8_t* spins_out, uint8_t* present_out, uint64_t* missing,
                                             uint64_t* external) {
    return guarded([&] {
        if (!spins_out || !present_out) throw wlg::WlgError(WLG_ERR_INVALID_ARGUMENT, "null argument");
        wlg::select_initial_configurations(emin, emax, width, windows, count, representative_energy,
                                           representative_spins, representative_present, representatives, spins,
                                           walkers_per_window, spins_out, present_out, missing, external);
    });
}

}  // extern "C"
