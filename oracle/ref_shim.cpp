// ref_shim.cpp — TEST INFRASTRUCTURE ONLY.
//
// A C-ABI wrapper around the *unmodified* reference library (Faikert/
// replica_exchange_wang_landau), compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/libwlref.so.  It lets the Python tests, the golden-
// fixture script and the CPU arm of bench.py call the reference's C++ API (physics
// helpers, WangLandauWalker, run_rewl, exact_enumeration) with the same POD types as the
// engine's C-ABI (include/wlg.h).  Nothing in the product links this file.
#include "wl/parallel.hpp"
#include "wl/analysis.hpp"
#include "wl/io.hpp"
#include "wl/physics.hpp"
#include "wl/wang_landau.hpp"

#include "../include/wlg.h"

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

void put_error(char* buffer, size_t size, const std::string& message) {
    if (!buffer || size == 0) return;
    const auto count = std::min(size - 1, message.size());
    std::memcpy(buffer, message.data(), count);
    buffer[count] = '\0';
}

wl::Geometry to_geometry(const wlg_system* s) {
    wl::Geometry g;
    g.box = {{s->box[0], s->box[1], s->box[2]}, s->periodic != 0};
    for (uint64_t i = 0; i < s->n; ++i) {
        g.positions.push_back({s->positions[3 * i], s->positions[3 * i + 1], s->positions[3 * i + 2]});
        g.axes.push_back({s->axes[3 * i], s->axes[3 * i + 1], s->axes[3 * i + 2]});
    }
    return g;
}

std::shared_ptr<const wl::Couplings> to_couplings(const wlg_system* s) {
    const auto g = to_geometry(s);
    if (s->cutoff > 0.0) return std::make_shared<wl::CsrCouplings>(g, s->coupling_scale, s->cutoff);
    return std::make_shared<wl::DenseCouplings>(g, s->coupling_scale);
}

wl::WlParameters to_parameters(const wlg_wl_parameters* p) {
    wl::WlParameters r;
    r.flatness = p->flatness;
    r.minimum_visits = p->minimum_visits;
    r.final_factor = p->final_factor;
    r.check_interval_attempts = p->check_interval_attempts;
    r.force_accept_after_attempts = p->force_accept_after_attempts;
    r.inverse_time_enabled = p->inverse_time_enabled != 0;
    r.initialization_max_attempts = p->initialization_max_attempts;
    r.initialization_target_fraction = p->initialization_target_fraction;
    r.initialization_temperature_fraction = p->initialization_temperature_fraction;
    r.initialization_stall_attempts_per_spin = p->initialization_stall_attempts_per_spin;
    r.initialization_temperature_multiplier = p->initialization_temperature_multiplier;
    r.initialization_max_temperature_fraction = p->initialization_max_temperature_fraction;
    r.collect_window_statistics = p->collect_window_statistics != 0;
    r.round_trip_margin_fraction = p->round_trip_margin_fraction;
    r.nalivaiko_mod = p->nalivaiko_mod != 0;
    return r;
}

struct WalkerHandle {
    std::shared_ptr<const wl::Couplings> couplings;
    std::unique_ptr<wl::WangLandauWalker> walker;
    std::size_t bins{};
};

struct ResultHandle {
    wl::RewlResult result;
    std::size_t bins{};
    std::size_t spins{};
};

int status_of(const std::exception& e) {
    if (dynamic_cast<const std::invalid_argument*>(&e)) return WLG_ERR_INVALID_ARGUMENT;
    if (dynamic_cast<const std::out_of_range*>(&e)) return WLG_ERR_OUT_OF_RANGE;
    if (dynamic_cast<const std::logic_error*>(&e)) return WLG_ERR_LOGIC;
    return WLG_ERR_RUNTIME;
}

} // namespace

extern "C" {

int ref_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

double ref_dipolar_pair(const double* d, const double* ai, const double* aj, double scale) {
    return wl::dipolar_pair({d[0], d[1], d[2]}, {ai[0], ai[1], ai[2]}, {aj[0], aj[1], aj[2]}, scale);
}

void ref_minimum_image(const double* d, const double* box, int periodic, double* out) {
    const auto r = wl::minimum_image({d[0], d[1], d[2]}, {{box[0], box[1], box[2]}, periodic != 0});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

int ref_grid_index(double emin, double emax, double width, double energy, int64_t* bin) {
    const wl::EnergyGrid grid{emin, emax, width};
    const auto b = grid.index(energy);
    *bin = b ? static_cast<int64_t>(*b) : -1;
    return 0;
}

int ref_partition_windows(uint64_t bins, uint64_t count, double overlap, uint64_t* out,
                          char* err, size_t errlen) {
    try {
        const auto w = wl::partition_windows(bins, count, overlap);
        for (std::size_t i = 0; i < w.size(); ++i) { out[2 * i] = w[i].begin; out[2 * i + 1] = w[i].end; }
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_couplings_dense(const wlg_system* s, double* out, char* err, size_t errlen) {
    try {
        const auto c = to_couplings(s);
        for (uint64_t i = 0; i < s->n; ++i)
            for (uint64_t j = 0; j < s->n; ++j) out[i * s->n + j] = c->at(i, j);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_fields(const wlg_system* s, const int8_t* spins, uint64_t count, double* fields,
               double* energies, char* err, size_t errlen) {
    try {
        const auto c = to_couplings(s);
        for (uint64_t k = 0; k < count; ++k) {
            const std::span<const std::int8_t> sp(spins + k * s->n, s->n);
            const auto f = wl::local_fields(*c, sp);
            std::copy(f.begin(), f.end(), fields + k * s->n);
            energies[k] = wl::total_energy(*c, sp);
        }
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_exact_enumeration(const wlg_system* s, double emin, double emax, double width,
                          uint64_t* counts, char* err, size_t errlen) {
    try {
        const auto c = to_couplings(s);
        const auto f = wl::exact_enumeration(*c, {emin, emax, width});
        std::copy(f.histogram.begin(), f.histogram.end(), counts);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

void* ref_walker_create(const wlg_system* s, uint64_t id, double emin, double emax, double width,
                        uint64_t window_begin, uint64_t window_end, const wlg_wl_parameters* p,
                        uint64_t seed, const int8_t* initial_spins, char* err, size_t errlen) {
    try {
        auto h = std::make_unique<WalkerHandle>();
        h->couplings = to_couplings(s);
        const wl::EnergyGrid grid{emin, emax, width};
        h->bins = grid.bins();
        std::vector<std::int8_t> spins;
        if (initial_spins) spins.assign(initial_spins, initial_spins + s->n);
        h->walker = std::make_unique<wl::WangLandauWalker>(
            id, h->couplings, grid, wl::EnergyWindow{window_begin, window_end}, to_parameters(p), seed,
            std::move(spins));
        return h.release();
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return nullptr; }
}

void ref_walker_destroy(void* handle) { delete static_cast<WalkerHandle*>(handle); }

int ref_walker_run(void* handle, uint64_t count, char* err, size_t errlen) {
    try { static_cast<WalkerHandle*>(handle)->walker->run_attempts(count); return 0; }
    catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_walker_attempt(void* handle, int* accepted, char* err, size_t errlen) {
    try { *accepted = static_cast<WalkerHandle*>(handle)->walker->attempt_flip() ? 1 : 0; return 0; }
    catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_walker_snapshot(void* handle, wlg_snapshot* out) {
    const auto s = static_cast<WalkerHandle*>(handle)->walker->snapshot();
    out->walker_id = s.walker_id;
    if (out->spins) std::copy(s.spins.begin(), s.spins.end(), out->spins);
    if (out->fields) std::copy(s.fields.begin(), s.fields.end(), out->fields);
    out->energy = s.energy;
    if (out->log_g) std::copy(s.log_g.begin(), s.log_g.end(), out->log_g);
    if (out->histogram) std::copy(s.histogram.begin(), s.histogram.end(), out->histogram);
    if (out->active) std::copy(s.active.begin(), s.active.end(), out->active);
    out->factor = s.factor;
    out->attempted = s.attempted;
    out->accepted = s.accepted;
    out->forced_accepted = s.forced_accepted;
    out->last_accepted_attempt = s.last_accepted_attempt;
    out->stage = static_cast<uint8_t>(s.stage);
    for (int k = 0; k < 4; ++k) out->rng_state[k] = s.rng_state[k];
    return 0;
}

int ref_walker_restore(void* handle, const wlg_snapshot* in, char* err, size_t errlen) {
    try {
        auto* h = static_cast<WalkerHandle*>(handle);
        const auto n = h->couplings->size();
        wl::WalkerSnapshot s;
        s.walker_id = in->walker_id;
        s.spins.assign(in->spins, in->spins + n);
        s.fields.assign(in->fields, in->fields + n);
        s.energy = in->energy;
        s.log_g.assign(in->log_g, in->log_g + h->bins);
        s.histogram.assign(in->histogram, in->histogram + h->bins);
        s.active.assign(in->active, in->active + h->bins);
        s.factor = in->factor;
        s.attempted = in->attempted;
        s.accepted = in->accepted;
        s.forced_accepted = in->forced_accepted;
        s.last_accepted_attempt = in->last_accepted_attempt;
        s.stage = static_cast<wl::RefinementStage>(in->stage);
        for (int k = 0; k < 4; ++k) s.rng_state[k] = in->rng_state[k];
        h->walker->restore(s);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

void ref_walker_histogram_statistics(void* handle, wlg_histogram_statistics* out) {
    const auto s = static_cast<WalkerHandle*>(handle)->walker->histogram_statistics();
    out->active_bins = s.active_bins;
    out->covered_bins = s.covered_bins;
    out->minimum = s.minimum;
    out->mean = s.mean;
    out->min_over_mean = s.min_over_mean;
    out->coverage = s.coverage;
}

void ref_walker_flags(void* handle, int* flat, int* covered, int* ready) {
    const auto& w = *static_cast<WalkerHandle*>(handle)->walker;
    *flat = w.flat() ? 1 : 0;
    *covered = w.covered() ? 1 : 0;
    *ready = w.ready_for_iteration() ? 1 : 0;
}

int ref_walker_begin_next_iteration(void* handle, char* err, size_t errlen) {
    try { static_cast<WalkerHandle*>(handle)->walker->begin_next_iteration(); return 0; }
    catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

double ref_walker_exchange_log_probability(void* left, void* right) {
    return static_cast<WalkerHandle*>(left)->walker->exchange_log_probability(
        *static_cast<WalkerHandle*>(right)->walker);
}

int ref_walker_swap(void* left, void* right, char* err, size_t errlen) {
    try {
        static_cast<WalkerHandle*>(left)->walker->swap_configuration(*static_cast<WalkerHandle*>(right)->walker);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

void ref_walker_counters(void* handle, uint64_t* out /* attempted, accepted, forced, last */) {
    const auto& w = *static_cast<WalkerHandle*>(handle)->walker;
    out[0] = w.attempted(); out[1] = w.accepted(); out[2] = w.forced_accepted(); out[3] = w.last_accepted_attempt();
}

// Walker-statistics arrays of the adaptive pilot (include/wl/wang_landau.hpp:118-127).
void ref_walker_pilot(void* handle, double* squared_displacement, uint64_t* samples,
                      uint64_t* round_trips, double* representative_energies,
                      int8_t* representative_spins, uint8_t* representative_present) {
    const auto& w = *static_cast<WalkerHandle*>(handle)->walker;
    const auto& sq = w.squared_energy_displacement();
    const auto& ds = w.displacement_samples();
    if (squared_displacement) std::copy(sq.begin(), sq.end(), squared_displacement);
    if (samples) std::copy(ds.begin(), ds.end(), samples);
    *round_trips = w.round_trips();
    const auto& reps = w.representatives();
    for (std::size_t r = 0; r < reps.size(); ++r) {
        representative_energies[r] = reps[r].energy;
        representative_present[r] = reps[r].spins.empty() ? 0 : 1;
        if (!reps[r].spins.empty())
            std::copy(reps[r].spins.begin(), reps[r].spins.end(),
                      representative_spins + r * reps[r].spins.size());
    }
}

void* ref_run_rewl(const wlg_system* s, const wlg_run_config* c, char* err, size_t errlen) {
    try {
        int argc = 1;
        char name[] = "ref";
        char* args[] = {name, nullptr};
        char** argv = args;
        wl::ParallelContext context(argc, argv);
        auto couplings = to_couplings(s);
        wl::RunConfig config;
        config.nx = config.ny = config.nz = 1;
        config.grid = {c->emin, c->emax, c->bin_width};
        config.energy_grid_explicit = true;
        config.windows = c->windows;
        config.walkers_per_rank = c->walkers_per_window;
        config.overlap = c->overlap;
        if (c->explicit_windows)
            for (uint64_t w = 0; w < c->windows; ++w)
                config.explicit_windows.push_back({c->explicit_windows[2 * w], c->explicit_windows[2 * w + 1]});
        config.seed = c->seed;
        config.seed_explicit = true;
        config.wl = to_parameters(&c->wl);
        config.exchange_interval_attempts = c->exchange_interval_attempts;
        config.max_attempts = c->max_attempts;
        config.checkpoint_interval_attempts = c->checkpoint_interval_attempts;
        if (c->checkpoint_path) config.checkpoint_path = c->checkpoint_path;
        config.progress_interval_seconds = c->progress_interval_seconds;
        if (c->initial_spins) {
            const auto total = c->windows * c->walkers_per_window;
            for (uint64_t w = 0; w < total; ++w) {
                if (c->initial_spins_present && !c->initial_spins_present[w]) config.initial_spins_by_walker.emplace_back();
                else config.initial_spins_by_walker.emplace_back(c->initial_spins + w * s->n, c->initial_spins + (w + 1) * s->n);
            }
        }
        auto h = std::make_unique<ResultHandle>();
        h->bins = config.grid.bins();
        h->spins = s->n;
        h->result = wl::run_rewl(context, couplings, config);
        return h.release();
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return nullptr; }
}

void ref_result_destroy(void* handle) { delete static_cast<ResultHandle*>(handle); }

void ref_result_totals(void* handle, wlg_run_totals* out) {
    const auto& r = static_cast<ResultHandle*>(handle)->result;
    out->attempted = r.attempted; out->accepted = r.accepted; out->forced_accepted = r.forced_accepted;
    out->exchange_attempted = r.exchange_attempted; out->exchange_accepted = r.exchange_accepted;
    out->converged = r.converged ? 1 : 0; out->epochs = 0;
}

int ref_result_fragment(void* handle, uint64_t w, double* log_g, uint64_t* histogram,
                        double* standard_error, uint8_t* valid) {
    const auto& r = static_cast<ResultHandle*>(handle)->result;
    if (w >= r.fragments.size()) return WLG_ERR_OUT_OF_RANGE;
    const auto& f = r.fragments[w];
    std::copy(f.log_g.begin(), f.log_g.end(), log_g);
    std::copy(f.histogram.begin(), f.histogram.end(), histogram);
    std::copy(f.standard_error.begin(), f.standard_error.end(), standard_error);
    std::copy(f.valid.begin(), f.valid.end(), valid);
    return 0;
}

uint64_t ref_result_walker_statistics(void* handle, wlg_walker_statistics* out, uint64_t capacity) {
    const auto& r = static_cast<ResultHandle*>(handle)->result;
    const auto count = std::min<uint64_t>(capacity, r.walker_statistics.size());
    for (uint64_t k = 0; k < count; ++k) {
        const auto& s = r.walker_statistics[k];
        out[k] = {s.walker_id, s.window_id, s.mpi_rank, s.attempted, s.accepted, s.forced_accepted,
                  s.attempts_since_last_accepted, s.energy, s.factor, s.active_bins, s.minimum_histogram,
                  s.mean_histogram, s.min_over_mean, s.round_trips};
    }
    return r.walker_statistics.size();
}

int ref_result_sampling(void* handle, uint64_t w, double* squared_displacement, uint64_t* samples,
                        uint64_t* round_trips, uint64_t* walkers) {
    const auto& r = static_cast<ResultHandle*>(handle)->result;
    if (w >= r.sampling_statistics.size()) return WLG_ERR_OUT_OF_RANGE;
    const auto& s = r.sampling_statistics[w];
    std::copy(s.squared_energy_displacement.begin(), s.squared_energy_displacement.end(), squared_displacement);
    std::copy(s.displacement_samples.begin(), s.displacement_samples.end(), samples);
    *round_trips = s.round_trips;
    *walkers = s.walkers;
    return 0;
}

uint64_t ref_result_representatives(void* handle, double* energies, int8_t* spins, uint64_t capacity) {
    const auto* h = static_cast<ResultHandle*>(handle);
    const auto& reps = h->result.representatives;
    const auto count = std::min<uint64_t>(capacity, reps.size());
    for (uint64_t k = 0; k < count; ++k) {
        energies[k] = reps[k].energy;
        std::copy(reps[k].spins.begin(), reps[k].spins.end(), spins + k * h->spins);
    }
    return reps.size();
}

// adapt_energy_windows + select_adaptive_initial_configurations are host post-processing
// (src/analysis.cpp:183-420); exposed so the adaptive pilot can be cross-checked.
int ref_adapt_windows(void* handle, double emin, double emax, double width, uint64_t count,
                      double overlap, uint64_t* out, char* err, size_t errlen) {
    try {
        const auto& r = static_cast<ResultHandle*>(handle)->result;
        const auto w = wl::adapt_energy_windows({emin, emax, width}, r.fragments, r.sampling_statistics,
                                                count, overlap, wl::AdaptiveWindowParameters{});
        for (std::size_t i = 0; i < w.size(); ++i) { out[2 * i] = w[i].begin; out[2 * i + 1] = w[i].end; }
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

// wl::stitch_dos and the DOS / fragment writers (src/analysis.cpp:45-130, src/io.cpp:398-421),
// for the byte-level comparison of the stitched output.
static std::vector<wl::DosFragment> fragments_from(const wlg_fragment_view* f, uint64_t count, uint64_t bins) {
    std::vector<wl::DosFragment> out(count);
    for (uint64_t k = 0; k < count; ++k) {
        out[k].window = {f[k].window_begin, f[k].window_end};
        out[k].log_g.assign(f[k].log_g, f[k].log_g + bins);
        out[k].histogram.assign(f[k].histogram, f[k].histogram + bins);
        out[k].standard_error.assign(f[k].standard_error, f[k].standard_error + bins);
        out[k].valid.assign(f[k].valid, f[k].valid + bins);
    }
    return out;
}

int ref_stitch_dos(double emin, double emax, double width, const wlg_fragment_view* f, uint64_t count, int complete,
                   uint64_t spins, double* lg, uint64_t* h, double* se, uint8_t* v, uint64_t* joins,
                   const char* dos_csv, char* err, size_t errlen) {
    try {
        const wl::EnergyGrid grid{emin, emax, width};
        const auto bins = grid.bins();
        const auto frags = fragments_from(f, count, bins);
        const auto dos = wl::stitch_dos(grid, frags, complete != 0, spins);
        std::copy(dos.log_g.begin(), dos.log_g.end(), lg);
        std::copy(dos.histogram.begin(), dos.histogram.end(), h);
        std::copy(dos.standard_error.begin(), dos.standard_error.end(), se);
        std::copy(dos.valid.begin(), dos.valid.end(), v);
        for (std::size_t k = 0; k < dos.join_bins.size(); ++k) joins[k] = dos.join_bins[k];
        if (dos_csv && dos_csv[0]) wl::write_dos_csv(dos_csv, dos);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_write_fragment_csv(const char* path, double emin, double emax, double width, const wlg_fragment_view* f,
                           uint64_t window_id, char* err, size_t errlen) {
    try {
        const wl::EnergyGrid grid{emin, emax, width};
        const auto frags = fragments_from(f, 1, grid.bins());
        wl::write_fragment_csv(path, grid, frags[0], window_id);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

// wl::write_workers_stat_csv (src/io.cpp:430-451) on wlg_walker_statistics rows.
int ref_write_workers_stat_csv(const char* path, const wlg_walker_statistics* s, uint64_t count, uint64_t spins,
                               char* err, size_t errlen) {
    try {
        std::vector<wl::WalkerStatistics> rows(count);
        for (uint64_t k = 0; k < count; ++k) {
            auto& r = rows[k];
            r.walker_id = s[k].walker_id;
            r.window_id = s[k].window_id;
            r.mpi_rank = s[k].mpi_rank;
            r.attempted = s[k].attempted;
            r.accepted = s[k].accepted;
            r.forced_accepted = s[k].forced_accepted;
            r.attempts_since_last_accepted = s[k].attempts_since_last_accepted;
            r.energy = s[k].energy;
            r.factor = s[k].factor;
            r.active_bins = s[k].active_bins;
            r.minimum_histogram = s[k].minimum_histogram;
            r.mean_histogram = s[k].mean_histogram;
            r.min_over_mean = s[k].min_over_mean;
            r.round_trips = s[k].round_trips;
        }
        wl::write_workers_stat_csv(path, rows, spins);
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

int ref_select_initial(void* handle, double emin, double emax, double width, const uint64_t* windows, uint64_t count,
                       uint64_t walkers, uint64_t n, int8_t* spins_out, uint8_t* present_out, uint64_t* missing,
                       uint64_t* external, char* err, size_t errlen) {
    try {
        const auto& r = static_cast<ResultHandle*>(handle)->result;
        std::vector<wl::EnergyWindow> w(count);
        for (uint64_t k = 0; k < count; ++k) w[k] = {windows[2 * k], windows[2 * k + 1]};
        std::size_t miss = 0, ext = 0;
        const auto seeds = wl::select_adaptive_initial_configurations({emin, emax, width}, w, r.representatives, 1,
                                                                      walkers, miss, ext);
        for (std::size_t k = 0; k < seeds.size(); ++k) {
            present_out[k] = seeds[k].empty() ? 0 : 1;
            if (!seeds[k].empty()) std::copy(seeds[k].begin(), seeds[k].end(), spins_out + k * n);
        }
        *missing = miss;
        *external = ext;
        return 0;
    } catch (const std::exception& e) { put_error(err, errlen, e.what()); return status_of(e); }
}

} // extern "C"
