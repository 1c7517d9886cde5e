// stitch.cpp — joining the windows' DOS fragments into one density of states, and the CSV
// writers of the DOS and of a fragment.
//
// stitch_dos follows wl::stitch_dos (src/analysis.cpp:45-130) operation for operation, on the
// host: the work is O(bins x windows), and the host C library's exp/log are the ones the
// reference uses, so the stitched curve is bit-identical.  The per-join overlap quality
// (common bins, RMSE and maximum deviation of the aligned curves, slope mismatch at the
// join) is an addition the reference does not report.  The writers follow write_dos_csv and
// write_fragment_csv (src/io.cpp:398-421): same header, same 17-significant-digit stream
// formatting, byte-compatible files.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <limits>
#include <numeric>
#include <vector>

#include "engine.hpp"

namespace wlg {

namespace {

constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

// log(sum exp(v)) over the finite entries; -inf when there are none.
double finite_log_sum_exp(const std::vector<double>& v) {
    double top = -std::numeric_limits<double>::infinity();
    for (double x : v)
        if (std::isfinite(x)) top = std::max(top, x);
    if (!std::isfinite(top)) return top;
    double sum = 0.0;
    for (double x : v)
        if (std::isfinite(x)) sum += std::exp(x - top);
    return top + std::log(sum);
}

// Least-squares slope of log g against the bin index over the five bins around `centre`
// (clipped to [begin, end)), valid and finite bins only, per unit energy; NaN below 2 points.
double slope_at(const std::vector<double>& lg, const std::vector<uint8_t>& ok, size_t centre, size_t begin, size_t end,
                double width) {
    const size_t lo = centre > 2 ? std::max(begin, centre - 2) : begin;
    const size_t hi = std::min(end, centre + 3);
    size_t points = 0;
    double sx = 0.0, sy = 0.0;
    for (size_t i = lo; i < hi; ++i)
        if (ok[i] != 0 && std::isfinite(lg[i])) {
            sx += static_cast<double>(i);
            sy += lg[i];
            ++points;
        }
    if (points < 2) return kNaN;
    sx /= static_cast<double>(points);
    sy /= static_cast<double>(points);
    double sxy = 0.0, sxx = 0.0;
    for (size_t i = lo; i < hi; ++i)
        if (ok[i] != 0 && std::isfinite(lg[i])) {
            const double dx = static_cast<double>(i) - sx;
            sxy += dx * (lg[i] - sy);
            sxx += dx * dx;
        }
    return sxx > 0.0 ? sxy / sxx / width : kNaN;
}

}  // namespace

void stitch_dos(double emin, double emax, double width, const wlg_fragment_view* in, uint64_t count,
                bool complete_range, uint64_t spins, double* out_lg, uint64_t* out_h, double* out_se, uint8_t* out_v,
                wlg_join_quality* joins, int32_t* fully_normalized) {
    validate_grid(emin, emax, width);
    if (count == 0 || !in) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "No DOS fragments supplied");
    const size_t bins = grid_bins(emin, emax, width);
    std::vector<wlg_fragment_view> frags(in, in + count);
    std::stable_sort(frags.begin(), frags.end(),
                     [](const wlg_fragment_view& a, const wlg_fragment_view& b) { return a.window_begin < b.window_begin; });
    for (const auto& f : frags)
        if (!f.log_g || !f.histogram || !f.standard_error || !f.valid || f.window_end > bins ||
            f.window_begin >= f.window_end)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "DOS fragment size mismatch");

    std::vector<double> lg(bins, kNaN), se(bins, kNaN);
    std::vector<uint64_t> h(bins, 0);
    std::vector<uint8_t> ok(bins, 0);
    const wlg_fragment_view& first = frags.front();
    for (size_t i = first.window_begin; i < first.window_end; ++i) {
        h[i] = first.histogram[i];
        ok[i] = first.valid[i];
        if (first.valid[i] != 0) {
            lg[i] = first.log_g[i];
            se[i] = first.standard_error[i];
        }
    }
    size_t covered = first.window_end;
    for (size_t f = 1; f < frags.size(); ++f) {
        const wlg_fragment_view& r = frags[f];
        if (r.window_begin >= covered)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "DOS fragments must overlap and match the global grid");
        const size_t ob = r.window_begin, oe = std::min(covered, static_cast<size_t>(r.window_end));
        // fallback join: the common valid bin nearest the middle of the overlap
        const size_t middle = ob + (oe - ob) / 2;
        size_t join = oe, nearest = std::numeric_limits<size_t>::max();
        for (size_t i = ob; i < oe; ++i)
            if (ok[i] != 0 && r.valid[i] != 0 && std::isfinite(lg[i]) && std::isfinite(r.log_g[i])) {
                const size_t d = i > middle ? i - middle : middle - i;
                if (d < nearest) {
                    nearest = d;
                    join = i;
                }
            }
        if (join == oe) throw WlgError(WLG_ERR_RUNTIME, "Adjacent DOS fragments have no common valid overlap bin");
        // preferred join: the bin where the two curves' local slopes agree best
        std::vector<double> right(r.log_g, r.log_g + bins);
        std::vector<uint8_t> right_ok(r.valid, r.valid + bins);
        double best = std::numeric_limits<double>::infinity();
        for (size_t i = ob + 2; i + 2 < oe; ++i) {
            if (ok[i] == 0 || right_ok[i] == 0) continue;
            const double d = std::abs(slope_at(lg, ok, i, ob, oe, width) - slope_at(right, right_ok, i, ob, oe, width));
            if (std::isfinite(d) && d < best) {
                best = d;
                join = i;
            }
        }
        const double shift = lg[join] - right[join];
        if (joins) {  // quality of the alignment over the whole overlap
            wlg_join_quality q{};
            q.join_bin = join;
            double s2 = 0.0, mx = 0.0;
            for (size_t i = ob; i < oe; ++i)
                if (ok[i] != 0 && right_ok[i] != 0 && std::isfinite(lg[i]) && std::isfinite(right[i])) {
                    const double d = lg[i] - (right[i] + shift);
                    s2 += d * d;
                    mx = std::max(mx, std::abs(d));
                    ++q.common_bins;
                }
            q.rmse = q.common_bins ? std::sqrt(s2 / static_cast<double>(q.common_bins)) : kNaN;
            q.max_abs_difference = mx;
            q.slope_difference = std::isfinite(best) ? best : kNaN;
            joins[f - 1] = q;
        }
        for (size_t i = join; i < r.window_end; ++i) {
            h[i] = r.histogram[i];
            ok[i] = r.valid[i];
            if (r.valid[i] != 0) {
                lg[i] = right[i] + shift;
                se[i] = r.standard_error[i];
            } else {
                lg[i] = kNaN;
                se[i] = kNaN;
            }
        }
        covered = std::max(covered, static_cast<size_t>(r.window_end));
    }
    if (complete_range) {
        if (std::any_of(ok.begin(), ok.end(), [](uint8_t v) { return v == 0; }))
            throw WlgError(WLG_ERR_RUNTIME, "Complete-range normalization requires every DOS bin to be valid");
        const double shift = static_cast<double>(spins) * std::log(2.0) - finite_log_sum_exp(lg);
        for (size_t i = 0; i < bins; ++i)
            if (ok[i] != 0) lg[i] += shift;
    } else {
        if (!std::isfinite(finite_log_sum_exp(lg))) throw WlgError(WLG_ERR_RUNTIME, "Stitched DOS has no valid bins");
        double peak = -std::numeric_limits<double>::infinity();
        for (size_t i = 0; i < bins; ++i)
            if (ok[i] != 0) peak = std::max(peak, lg[i]);
        for (size_t i = 0; i < bins; ++i)
            if (ok[i] != 0) lg[i] -= peak;
    }
    std::copy(lg.begin(), lg.end(), out_lg);
    std::copy(h.begin(), h.end(), out_h);
    std::copy(se.begin(), se.end(), out_se);
    std::copy(ok.begin(), ok.end(), out_v);
    if (fully_normalized) *fully_normalized = complete_range ? 1 : 0;
}

void write_dos_csv(const char* path, double emin, double width, uint64_t bins, const double* lg, const uint64_t* h,
                   const double* se, const uint8_t* ok) {
    std::ofstream out(path);
    if (!out) throw WlgError(WLG_ERR_IO, std::string("Cannot write ") + path);
    out << "bin,energy,log_g,histogram,standard_error,valid\n" << std::setprecision(17);
    for (uint64_t i = 0; i < bins; ++i)
        out << i << ',' << emin + (static_cast<double>(i) + 0.5) * width << ',' << lg[i] << ',' << h[i] << ','
            << se[i] << ',' << static_cast<unsigned>(ok[i]) << '\n';
}

void write_fragment_csv(const char* path, double emin, double width, uint64_t window_id, uint64_t begin,
                        uint64_t end, const double* lg, const uint64_t* h, const double* se, const uint8_t* ok) {
    std::ofstream out(path);
    if (!out) throw WlgError(WLG_ERR_IO, std::string("Cannot write ") + path);
    out << "window,bin,energy,log_g,histogram,standard_error,valid\n" << std::setprecision(17);
    for (uint64_t i = begin; i < end; ++i)
        out << window_id << ',' << i << ',' << emin + (static_cast<double>(i) + 0.5) * width << ',' << lg[i] << ','
            << h[i] << ',' << se[i] << ',' << static_cast<unsigned>(ok[i]) << '\n';
}

// <prefix>_workers_stat.csv (src/io.cpp:430-451): one row per walker; the MCS columns divide
// the attempt counts by the spin count, and the acceptance percentage is 0 for a walker that
// made no attempt.
void write_workers_stat_csv(const char* path, const wlg_walker_statistics* stats, uint64_t count,
                            uint64_t spin_count) {
    if (spin_count == 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Cannot write MCS statistics for zero spins");
    std::ofstream out(path);
    if (!out) throw WlgError(WLG_ERR_IO, std::string("Cannot write ") + path);
    out << "mpi_rank,window,walker_id,attempted_flips,attempted_mcs,accepted,forced_accepted,accepted_percent,"
           "attempts_since_last_accepted,mcs_since_last_accepted,energy,factor,active_bins,min_h,mean_h,"
           "min_over_mean,round_trips\n"
        << std::setprecision(17);
    const double spins = static_cast<double>(spin_count);
    for (uint64_t k = 0; k < count; ++k) {
        const wlg_walker_statistics& s = stats[k];
        const double percent =
            s.attempted == 0 ? 0.0 : 100.0 * static_cast<double>(s.accepted) / static_cast<double>(s.attempted);
        out << s.mpi_rank << ',' << s.window_id << ',' << s.walker_id << ',' << s.attempted << ','
            << static_cast<double>(s.attempted) / spins << ',' << s.accepted << ',' << s.forced_accepted << ','
            << percent << ',' << s.attempts_since_last_accepted << ','
            << static_cast<double>(s.attempts_since_last_accepted) / spins << ',' << s.energy << ',' << s.factor
            << ',' << s.active_bins << ',' << s.minimum_histogram << ',' << s.mean_histogram << ','
            << s.min_over_mean << ',' << s.round_trips << '\n';
    }
}

}  // namespace wlg
