// adaptive.cpp — the adaptive-window pilot's host steps: choosing the next energy windows
// from a pilot run's fragments and sampling statistics (adapt_energy_windows,
// src/analysis.cpp:183-339) and seeding every walker of the new windows from the pilot's
// representative configurations (select_adaptive_initial_configurations,
// src/analysis.cpp:341-420, single process).  Host work of O(bins) per pilot, evaluated in
// the reference's order (long double prefix sums, the same percentile selections) so that the
// windows and seeds are identical and the production run that follows is the reference's.
//
// Window placement: every bin gets the weight
//     round-trip penalty * (1 + curvature weight * normalised |d2 log g / dE2|)
//       / sqrt(max(local diffusivity, floor))
// where the local diffusivity is the mean squared accepted energy step around the bin; the
// cores split the cumulative weight into equal parts (each at least a minimum width), and
// every core is extended on both sides by overlap / (2 (1 - overlap)) of its width.
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "engine.hpp"

namespace wlg {

std::vector<uint64_t> adapt_energy_windows(double emin, double emax, double width, const wlg_fragment_view* frags,
                                           const wlg_sampling_view* sampling, uint64_t count, double overlap,
                                           const wlg_adaptive_parameters& p) {
    validate_grid(emin, emax, width);
    const size_t bins = grid_bins(emin, emax, width);
    if (count == 0 || count > bins || !frags || !sampling || overlap < 0.0 || overlap >= 1.0 ||
        !std::isfinite(p.diffusivity_floor_fraction) || !(p.diffusivity_floor_fraction > 0.0) ||
        !std::isfinite(p.curvature_weight) || p.curvature_weight < 0.0 || !std::isfinite(p.round_trip_target) ||
        p.round_trip_target < 0.0 || !std::isfinite(p.maximum_round_trip_penalty) ||
        p.maximum_round_trip_penalty < 1.0 || !std::isfinite(p.smoothing_width) || p.smoothing_width < 0.0 ||
        !std::isfinite(p.minimum_width) || p.minimum_width < 0.0)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid adaptive-window parameters");
    if (count == 1) return {0, bins};

    std::vector<double> disp(bins, 0.0), curv(bins, 0.0), penalty(bins, 1.0);
    std::vector<uint64_t> samples(bins, 0), curv_n(bins, 0);
    const double auto_smoothing = (emax - emin) / (10.0 * static_cast<double>(count));
    const double smoothing = std::max(width, p.smoothing_width > 0.0 ? p.smoothing_width : auto_smoothing);
    const size_t radius = std::max<size_t>(1, static_cast<size_t>(std::llround(smoothing / width)));

    for (uint64_t w = 0; w < count; ++w) {
        const wlg_sampling_view& s = sampling[w];
        const wlg_fragment_view& f = frags[w];
        if (s.window_begin != f.window_begin || s.window_end != f.window_end || s.window_end > bins ||
            !s.squared_energy_displacement || !s.displacement_samples || !f.log_g || !f.valid)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Adaptive-window pilot fragments are incompatible");
        for (size_t i = s.window_begin; i < s.window_end; ++i) {
            disp[i] += s.squared_energy_displacement[i];
            samples[i] += s.displacement_samples[i];
        }
        const double expected = p.round_trip_target * static_cast<double>(s.walkers);
        const double observed = static_cast<double>(s.round_trips);
        const double pen = expected <= 0.0 ? 1.0
                                           : std::min(p.maximum_round_trip_penalty,
                                                      std::sqrt(expected / std::max(1.0, observed)));
        for (size_t i = s.window_begin; i < s.window_end; ++i) penalty[i] = std::max(penalty[i], pen);
        for (size_t i = f.window_begin + radius; i + radius < f.window_end; ++i) {
            if (f.valid[i - radius] == 0 || f.valid[i] == 0 || f.valid[i + radius] == 0) continue;
            const double h = static_cast<double>(radius) * width;
            const double c = std::abs(f.log_g[i + radius] - 2.0 * f.log_g[i] + f.log_g[i - radius]) / (h * h);
            if (std::isfinite(c)) {
                curv[i] += c;
                ++curv_n[i];
            }
        }
    }

    // local diffusivity: windowed mean of the squared steps (long double prefix sums)
    std::vector<long double> pd(bins + 1, 0.0L);
    std::vector<uint64_t> pn(bins + 1, 0);
    for (size_t i = 0; i < bins; ++i) {
        pd[i + 1] = pd[i] + disp[i];
        pn[i + 1] = pn[i] + samples[i];
    }
    std::vector<double> diff(bins, 0.0), positive;
    positive.reserve(bins);
    for (size_t i = 0; i < bins; ++i) {
        const size_t lo = i > radius ? i - radius : 0, hi = std::min(bins, i + radius + 1);
        const uint64_t n = pn[hi] - pn[lo];
        if (n != 0) diff[i] = static_cast<double>((pd[hi] - pd[lo]) / static_cast<long double>(n));
        if (diff[i] > 0.0 && std::isfinite(diff[i])) positive.push_back(diff[i]);
    }
    double typical = 1.0;
    if (!positive.empty()) {  // the median (upper middle) of the positive diffusivities
        auto mid = positive.begin() + static_cast<std::ptrdiff_t>(positive.size() / 2);
        std::nth_element(positive.begin(), mid, positive.end());
        typical = *mid;
    }
    const double floor_d = std::max(std::numeric_limits<double>::min(), p.diffusivity_floor_fraction * typical);

    std::vector<double> curv_pos;
    curv_pos.reserve(bins);
    for (size_t i = 0; i < bins; ++i)
        if (curv_n[i] != 0) {
            curv[i] /= static_cast<double>(curv_n[i]);
            if (curv[i] > 0.0 && std::isfinite(curv[i])) curv_pos.push_back(curv[i]);
        }
    double curv_scale = 1.0;
    if (!curv_pos.empty()) {  // the 90th percentile of the positive curvatures
        const size_t at = std::min(curv_pos.size() - 1, static_cast<size_t>(0.9 * static_cast<double>(curv_pos.size())));
        auto q = curv_pos.begin() + static_cast<std::ptrdiff_t>(at);
        std::nth_element(curv_pos.begin(), q, curv_pos.end());
        curv_scale = std::max(*q, std::numeric_limits<double>::min());
    }

    std::vector<long double> cw(bins + 1, 0.0L);
    for (size_t i = 0; i < bins; ++i) {
        const double nc = std::min(1.0, curv[i] / curv_scale);
        const double weight = penalty[i] * (1.0 + p.curvature_weight * nc) / std::sqrt(std::max(diff[i], floor_d));
        cw[i + 1] = cw[i] + static_cast<long double>(weight * width);
    }
    const long double total = cw.back();
    if (!(total > 0.0L)) throw WlgError(WLG_ERR_RUNTIME, "Adaptive-window weight is empty");

    const double span = emax - emin;
    const double min_width = p.minimum_width > 0.0 ? p.minimum_width : span / (4.0 * static_cast<double>(count));
    if (!(min_width > 0.0) || min_width * static_cast<double>(count) > span)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Adaptive minimum window width is too large");
    const size_t min_cells = std::max<size_t>(1, static_cast<size_t>(std::ceil(min_width / width)));

    std::vector<size_t> core(count + 1, 0);
    core.back() = bins;
    for (uint64_t k = 1; k < count; ++k) {
        const long double target = total * static_cast<long double>(k) / static_cast<long double>(count);
        size_t c = static_cast<size_t>(std::lower_bound(cw.begin(), cw.end(), target) - cw.begin());
        c = std::clamp(c, core[k - 1] + min_cells, bins - (count - k) * min_cells);
        core[k] = c;
    }
    const double extension = overlap == 0.0 ? 0.0 : overlap / (2.0 * (1.0 - overlap));
    std::vector<uint64_t> out(2 * count);
    for (uint64_t k = 0; k < count; ++k) {
        const size_t core_width = core[k + 1] - core[k];
        const size_t extra = static_cast<size_t>(std::ceil(extension * static_cast<double>(core_width)));
        out[2 * k] = k == 0 ? 0 : (core[k] > extra ? core[k] - extra : 0);
        out[2 * k + 1] = k + 1 == count ? bins : std::min(bins - (count - 1 - k), core[k + 1] + extra);
    }
    for (uint64_t k = 1; k < count; ++k) {
        out[2 * k] = std::max(out[2 * k], out[2 * (k - 1)] + 1);
        out[2 * k + 1] = std::max(out[2 * k + 1], out[2 * (k - 1) + 1] + 1);
        if (out[2 * k] >= out[2 * (k - 1) + 1] || out[2 * k] >= out[2 * k + 1])
            throw WlgError(WLG_ERR_RUNTIME, "Adaptive energy windows do not overlap");
    }
    return out;
}

// Seeds for every walker of the new windows (one process): the walkers of the lowest window
// all start from the lowest-energy representative; every other window takes, round robin,
// the representatives inside it ordered by distance to the window centre (or, when none is
// inside, all of them ordered by distance to the window, counted as external).
void select_initial_configurations(double emin, double emax, double width, const uint64_t* windows, uint64_t count,
                                   const double* rep_energy, const int8_t* rep_spins, const uint8_t* rep_present,
                                   uint64_t reps, uint64_t n, uint64_t walkers_per_window, int8_t* spins_out,
                                   uint8_t* present_out, uint64_t* missing, uint64_t* external) {
    validate_grid(emin, emax, width);
    if (count == 0 || walkers_per_window == 0 || !windows || (reps && (!rep_energy || !rep_spins || !rep_present)))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid adaptive initial-configuration layout");
    const Grid g = make_grid(emin, emax, width, static_cast<int64_t>(grid_bins(emin, emax, width)));
    uint64_t n_missing = 0, n_external = 0;
    int64_t lowest = -1;
    for (uint64_t r = 0; r < reps; ++r)
        if (rep_present[r] && (lowest < 0 || rep_energy[r] < rep_energy[lowest])) lowest = static_cast<int64_t>(r);
    auto assign = [&](uint64_t walker, int64_t r) {
        std::copy(rep_spins + static_cast<size_t>(r) * n, rep_spins + static_cast<size_t>(r + 1) * n,
                  spins_out + walker * n);
        present_out[walker] = 1;
    };
    for (uint64_t w = 0; w < count; ++w) {
        const uint64_t b = windows[2 * w], e = windows[2 * w + 1];
        const double lower = emin + static_cast<double>(b) * width, upper = emin + static_cast<double>(e) * width;
        const double centre = 0.5 * (lower + upper);
        for (uint64_t k = 0; k < walkers_per_window; ++k) present_out[w * walkers_per_window + k] = 0;
        if (w == 0 && lowest >= 0) {
            const int64_t bin = grid_index(g, rep_energy[lowest]);
            const bool outside = bin < 0 || static_cast<uint64_t>(bin) < b || static_cast<uint64_t>(bin) >= e;
            for (uint64_t k = 0; k < walkers_per_window; ++k) {
                assign(w * walkers_per_window + k, lowest);
                if (outside) ++n_external;
            }
            continue;
        }
        std::vector<int64_t> cand;
        for (uint64_t r = 0; r < reps; ++r) {
            if (!rep_present[r]) continue;
            const int64_t bin = grid_index(g, rep_energy[r]);
            if (bin >= 0 && static_cast<uint64_t>(bin) >= b && static_cast<uint64_t>(bin) < e)
                cand.push_back(static_cast<int64_t>(r));
        }
        const bool outside = cand.empty();
        if (outside)
            for (uint64_t r = 0; r < reps; ++r)
                if (rep_present[r]) cand.push_back(static_cast<int64_t>(r));
        auto gap = [lower, upper](double x) { return x < lower ? lower - x : (x >= upper ? x - upper : 0.0); };
        std::sort(cand.begin(), cand.end(), [&](int64_t a, int64_t c) {
            const double ga = gap(rep_energy[a]), gc = gap(rep_energy[c]);
            if (ga != gc) return ga < gc;
            const double da = std::abs(rep_energy[a] - centre), dc = std::abs(rep_energy[c] - centre);
            return da == dc ? rep_energy[a] < rep_energy[c] : da < dc;
        });
        for (uint64_t k = 0; k < walkers_per_window; ++k) {
            if (cand.empty()) {
                ++n_missing;
                continue;
            }
            assign(w * walkers_per_window + k, cand[k % cand.size()]);
            if (outside) ++n_external;
        }
    }
    if (missing) *missing = n_missing;
    if (external) *external = n_external;
}

}  // namespace wlg
