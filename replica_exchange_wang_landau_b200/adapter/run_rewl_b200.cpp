// run_rewl_b200.cpp — run_rewl (src/parallel.cpp:276-580) served by the B200 engine.
//
// Built against the reference's headers and linked with its io/analysis objects (for
// RunConfig::validate) and with libwlg.so.  See run_rewl_b200.hpp for the contract.
#include "run_rewl_b200.hpp"

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <utility>
#include <stdexcept>
#include <string>
#include <vector>

#include "wlg.h"

namespace wl {
namespace {

// wlg_status -> the exception type the reference throws for that condition.
void check(wlg_status status) {
    if (status == WLG_OK) return;
    const std::string message = wlg_last_error();
    switch (status) {
        case WLG_ERR_INVALID_ARGUMENT: throw std::invalid_argument(message);
        case WLG_ERR_LOGIC: throw std::logic_error(message);
        case WLG_ERR_OUT_OF_RANGE: throw std::out_of_range(message);
        default: throw std::runtime_error(message);
    }
}

struct EngineHandle {
    wlg_engine* engine = nullptr;
    ~EngineHandle() { wlg_engine_destroy(engine); }
};

// The couplings as Couplings::at(i, j) reads them.  Dense: the whole matrix.  CSR: the
// non-zero couplings of each row in column order (a stored coupling whose value is exactly
// zero is indistinguishable from an absent one through at(), and adds nothing to any field).
struct ExportedCouplings {
    std::vector<double> dense;
    std::vector<std::uint64_t> offsets, columns;
    std::vector<double> values;
    wlg_couplings view{};
};

void export_couplings(const Couplings& couplings, ExportedCouplings& out) {
    const std::size_t n = couplings.size();
    out.view.n = n;
    if (couplings.backend_name() != "csr") {
        out.dense.resize(n * n);
        #pragma omp parallel for schedule(static)
        for (std::int64_t ii = 0; ii < static_cast<std::int64_t>(n); ++ii) {
            const auto i = static_cast<std::size_t>(ii);
            for (std::size_t j = 0; j < n; ++j) out.dense[i * n + j] = couplings.at(i, j);
        }
        out.view.dense = out.dense.data();
        return;
    }
    std::vector<std::vector<std::pair<std::uint64_t, double>>> rows(n);
    #pragma omp parallel for schedule(dynamic, 64)
    for (std::int64_t ii = 0; ii < static_cast<std::int64_t>(n); ++ii) {
        const auto i = static_cast<std::size_t>(ii);
        for (std::size_t j = 0; j < n; ++j) {
            const double v = couplings.at(i, j);
            if (v != 0.0) rows[i].emplace_back(j, v);
        }
    }
    out.offsets.assign(n + 1, 0);
    for (std::size_t i = 0; i < n; ++i) out.offsets[i + 1] = out.offsets[i] + rows[i].size();
    out.columns.reserve(out.offsets[n]);
    out.values.reserve(out.offsets[n]);
    for (const auto& row : rows)
        for (const auto& [column, value] : row) {
            out.columns.push_back(column);
            out.values.push_back(value);
        }
    out.view.nnz = out.offsets[n];
    out.view.row_offsets = out.offsets.data();
    out.view.columns = out.columns.data();
    out.view.values = out.values.data();
}

}  // namespace

RewlResult run_rewl_b200(const ParallelContext& context, std::shared_ptr<const Couplings> couplings,
                         const RunConfig& c) {
    // the reference's own checks, in its order (src/parallel.cpp:278-294)
    if (!couplings) throw std::invalid_argument("Null couplings");
    c.validate(!c.smoke_test);
    if (context.size() > 1)
        throw std::invalid_argument("run_rewl_b200 drives one GPU per process; run it with one MPI rank");
    const std::size_t n = couplings->size();
    const std::size_t total = c.windows * c.walkers_per_rank;
    if (!c.initial_spins_by_walker.empty()) {
        if (c.initial_spins_by_walker.size() != total)
            throw std::invalid_argument("Adaptive initial-configuration count mismatch");
        for (const auto& spins : c.initial_spins_by_walker)
            if (!spins.empty() && spins.size() != n) throw std::invalid_argument("Adaptive initial spin count mismatch");
    }

    wlg_run_config rc{};
    rc.emin = c.grid.minimum;
    rc.emax = c.grid.maximum;
    rc.bin_width = c.grid.width;
    rc.windows = c.windows;
    rc.walkers_per_window = c.walkers_per_rank;
    rc.overlap = c.overlap;
    std::vector<std::uint64_t> windows;
    if (!c.explicit_windows.empty()) {
        for (const auto& w : c.explicit_windows) {
            windows.push_back(w.begin);
            windows.push_back(w.end);
        }
        if (windows.size() != 2 * c.windows)
            throw std::invalid_argument("Explicit energy windows must match the configured window count");
        rc.explicit_windows = windows.data();
    }
    rc.seed = c.seed;
    rc.wl.flatness = c.wl.flatness;
    rc.wl.minimum_visits = c.wl.minimum_visits;
    rc.wl.final_factor = c.wl.final_factor;
    rc.wl.check_interval_attempts = c.wl.check_interval_attempts;
    rc.wl.force_accept_after_attempts = c.wl.force_accept_after_attempts;
    rc.wl.inverse_time_enabled = c.wl.inverse_time_enabled ? 1 : 0;
    rc.wl.initialization_max_attempts = c.wl.initialization_max_attempts;
    rc.wl.initialization_target_fraction = c.wl.initialization_target_fraction;
    rc.wl.initialization_temperature_fraction = c.wl.initialization_temperature_fraction;
    rc.wl.initialization_stall_attempts_per_spin = c.wl.initialization_stall_attempts_per_spin;
    rc.wl.initialization_temperature_multiplier = c.wl.initialization_temperature_multiplier;
    rc.wl.initialization_max_temperature_fraction = c.wl.initialization_max_temperature_fraction;
    rc.wl.collect_window_statistics = c.wl.collect_window_statistics ? 1 : 0;
    rc.wl.round_trip_margin_fraction = c.wl.round_trip_margin_fraction;
    rc.wl.nalivaiko_mod = c.wl.nalivaiko_mod ? 1 : 0;
    rc.exchange_interval_attempts = c.exchange_interval_attempts;
    rc.max_attempts = c.max_attempts;
    rc.checkpoint_interval_attempts = c.checkpoint_interval_attempts;
    rc.checkpoint_path = c.checkpoint_path.empty() ? nullptr : c.checkpoint_path.c_str();
    std::vector<std::int8_t> spins;
    std::vector<std::uint8_t> present;
    if (!c.initial_spins_by_walker.empty()) {
        spins.assign(total * n, 1);
        present.assign(total, 0);
        for (std::size_t w = 0; w < total; ++w) {
            const auto& s = c.initial_spins_by_walker[w];
            if (s.empty()) continue;
            std::copy(s.begin(), s.end(), spins.begin() + static_cast<std::ptrdiff_t>(w * n));
            present[w] = 1;
        }
        rc.initial_spins = spins.data();
        rc.initial_spins_present = present.data();
    }
    rc.progress_interval_seconds = c.progress_interval_seconds;
    rc.coupling_precision = WLG_PRECISION_FP64;
    rc.recompute_interval_attempts = 0;

    ExportedCouplings exported;
    export_couplings(*couplings, exported);
    EngineHandle handle;
    check(wlg_engine_create_from_couplings(&exported.view, &rc, &handle.engine));
    wlg_run_totals totals{};
    check(wlg_engine_run(handle.engine, &totals));

    RewlResult result;
    const std::size_t bins = c.grid.bins();
    const bool collect = c.wl.collect_window_statistics;
    std::vector<wlg_walker_statistics> stats(total);
    check(wlg_engine_walker_statistics(handle.engine, stats.data(), total));
    for (const auto& s : stats)
        result.walker_statistics.push_back({s.walker_id, s.window_id, context.rank(), s.attempted, s.accepted,
                                            s.forced_accepted, s.attempts_since_last_accepted, s.energy, s.factor,
                                            static_cast<std::size_t>(s.active_bins), s.minimum_histogram,
                                            s.mean_histogram, s.min_over_mean, s.round_trips});
    if (collect) {
        const std::uint64_t capacity = total * 9;  // a walker's bank holds 9 representatives
        std::vector<double> energies(capacity);
        std::vector<std::int8_t> bank(capacity * n);
        std::uint64_t count = 0;
        check(wlg_engine_representatives(handle.engine, energies.data(), bank.data(), capacity, &count));
        for (std::uint64_t r = 0; r < count; ++r)
            result.representatives.push_back(
                {energies[r], std::vector<std::int8_t>(bank.begin() + static_cast<std::ptrdiff_t>(r * n),
                                                       bank.begin() + static_cast<std::ptrdiff_t>((r + 1) * n))});
    }
    std::vector<double> log_g(c.windows * bins), sem(c.windows * bins);
    std::vector<std::uint64_t> histogram(c.windows * bins);
    std::vector<std::uint8_t> valid(c.windows * bins);
    check(wlg_engine_fragments(handle.engine, collect ? 1 : 0, log_g.data(), histogram.data(), sem.data(),
                               valid.data()));
    for (std::size_t w = 0; w < c.windows; ++w) {
        std::uint64_t begin = 0, end = 0;
        check(wlg_engine_window(handle.engine, w, &begin, &end));
        const auto at = [&](auto& v) {
            return std::vector<typename std::decay_t<decltype(v)>::value_type>(
                v.begin() + static_cast<std::ptrdiff_t>(w * bins), v.begin() + static_cast<std::ptrdiff_t>((w + 1) * bins));
        };
        result.fragments.push_back({EnergyWindow{begin, end}, at(log_g), at(histogram), at(sem), at(valid)});
        if (collect) {
            WindowSamplingStatistics s{EnergyWindow{begin, end}, std::vector<double>(bins, 0.0),
                                       std::vector<std::uint64_t>(bins, 0), 0, 0};
            check(wlg_engine_sampling_statistics(handle.engine, w, s.squared_energy_displacement.data(),
                                                 s.displacement_samples.data(), &s.round_trips, &s.walkers));
            result.sampling_statistics.push_back(std::move(s));
        }
    }
    result.attempted = totals.attempted;
    result.accepted = totals.accepted;
    result.forced_accepted = totals.forced_accepted;
    result.exchange_attempted = totals.exchange_attempted;
    result.exchange_accepted = totals.exchange_accepted;
    result.converged = totals.converged != 0;
    return result;
}

}  // namespace wl
