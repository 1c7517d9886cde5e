// walker_dev.cuh — warp-level pieces of WangLandauWalker used by several kernels.
//
// A walker is owned by one warp.  All 32 lanes evaluate the walker's scalar chain
// redundantly (identical registers, no divergence, no shuffles on the hot path); the
// lanes split only the O(N) / O(z) field updates and the O(bins) histogram reductions.
// Shared-memory writes of scalars are done by lane 0 and published with __syncwarp().
#pragma once

#include "common.cuh"

namespace wlg {

constexpr unsigned kFull = 0xffffffffu;

// The acceptance test of attempt_flip and of the initialisation search,
// log(max(u, 2^-53)) < threshold (src/wang_landau.cpp:207-208, 261), with the same result
// as evaluating it with the full-precision log().  A one-instruction log2 estimate (MUFU)
// decides whenever it is farther than 1e-3 from the threshold: for u' in [2^-53, 1) its
// error, including the rounding of u' to float and of the product by ln 2, is below 1e-5,
// and log() itself is within one ulp, so the comparison cannot flip.  Only the ~0.1% of
// draws inside the margin pay for log().
__device__ __forceinline__ bool log_uniform_below(double u, double threshold) {
    const double up = fmax(u, 0x1.0p-53);
    const double estimate = static_cast<double>(__log2f(static_cast<float>(up))) * 0.6931471805599453;
    if (estimate < threshold - 1e-3) return true;
    if (estimate > threshold + 1e-3) return false;
    return log(up) < threshold;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const uint64_t y = __shfl_xor_sync(kFull, x, o);
        x = y < x ? y : x;
    }
    return x;
}

// histogram_statistics (src/wang_landau.cpp:344-367) over the window slice [0, nbins) of
// h / mask.  active_bins is the walker's cached counter, as in the reference.
struct HistStats {
    uint64_t active_bins;
    uint64_t covered;
    uint64_t minimum;
    double mean;
    double min_over_mean;
    double coverage;
};

__device__ __forceinline__ HistStats warp_histogram_statistics(const uint64_t* h, const uint8_t* mask, int nbins,
                                                               uint64_t active_bins, int lane) {
    uint64_t covered = 0, mn = ~0ULL, total = 0;
    for (int b = lane; b < nbins; b += 32) {
        if (!mask[b]) continue;
        const uint64_t v = h[b];
        covered += v != 0 ? 1 : 0;
        mn = v < mn ? v : mn;
        total += v;
    }
    covered = warp_sum_u64(covered);
    mn = warp_min_u64(mn);
    total = warp_sum_u64(total);
    HistStats s;
    s.active_bins = active_bins;
    s.covered = covered;
    s.minimum = mn;
    s.mean = 0.0;
    s.min_over_mean = 0.0;
    s.coverage = 0.0;
    if (active_bins == 0) {
        s.minimum = 0;
        return s;
    }
    s.mean = x87_mean(total, active_bins);
    s.min_over_mean = s.mean > 0.0 ? static_cast<double>(s.minimum) / s.mean : 0.0;
    s.coverage = static_cast<double>(covered) / static_cast<double>(active_bins);
    return s;
}

// flat / covered / ready_for_iteration (src/wang_landau.cpp:369-387)
__device__ __forceinline__ bool stats_flat(const HistStats& s, int32_t stage, const DeviceParams& p) {
    if (stage != kWangLandau) return true;
    return s.active_bins != 0 && s.minimum >= p.minimum_visits && s.min_over_mean >= p.flatness;
}
__device__ __forceinline__ bool stats_covered(const HistStats& s, int32_t stage) {
    if (stage != kWangLandau) return true;
    return s.active_bins != 0 && s.covered == s.active_bins;
}
__device__ __forceinline__ bool stats_ready(const HistStats& s, int32_t stage, const DeviceParams& p) {
    return stage == kWangLandau && (p.inverse_time ? stats_covered(s, stage) : stats_flat(s, stage, p));
}

// begin_next_iteration + freeze_if_finished (src/wang_landau.cpp:389-413); the caller has
// checked readiness.  h / refine are the window slices.
__device__ __forceinline__ void warp_begin_next_iteration(WalkerState& st, uint64_t* h, uint8_t* refine, int nbins,
                                                          const DeviceParams& p, int lane) {
    st.factor *= 0.5;
    for (int b = lane; b < nbins; b += 32) h[b] = 0;
    if (p.nalivaiko) {
        for (int b = lane; b < nbins; b += 32) refine[b] = 0;
        st.refine_count = 0;
    }
    if (p.inverse_time) {
        if (st.time_offset == kContinueSchedule) {
            // a warm start continuing the schedule: the 1/t stage starts at this check from the
            // factor reached, as if round(active / factor) attempts had been made
            const double made = fmin(nearbyint(static_cast<double>(st.active_count) / st.factor), 0x1.0p62);
            const double attempted = static_cast<double>(st.attempted);
            st.time_offset = made > attempted ? static_cast<uint64_t>(made - attempted) : 0;
            st.stage = kInverseTime;
        } else {
            const double inverse_time = st.attempted == 0 ? 1.0
                                                          : static_cast<double>(st.active_count) /
                                                                static_cast<double>(st.attempted + st.time_offset);
            if (st.factor <= inverse_time) {
                st.stage = kInverseTime;
                st.factor = inverse_time;
            }
        }
    }
    if (st.factor <= p.final_factor) st.stage = kFrozen;
    __syncwarp();
}

// update_inverse_time_factor (src/wang_landau.cpp:300-315) for consecutive attempts of the 1/t
// stage: f = active_bins / attempted, the attempted count including the attempt (plus the
// walker's time_offset, 0 unless a warm start continues the schedule).  An IEEE
// division is a dependent sequence of about 170 cycles that the warp would otherwise wait for
// on every attempt; here lane j divides for the j-th attempt of a block of 32 (the same
// operands, so the same quotient), and an attempt takes its quotient by a shuffle.  A block
// is recomputed after 32 attempts or when the active-bin count has changed.  With no active
// bin the factor is left unchanged, as the reference leaves it.  (Reading the quotient by a
// shuffle issued at the start of the attempt was measured slower.)
struct InverseTimeTable {
    double q = 0.0;        // lane j: active / (first + j + 1)
    uint64_t active = 0;   // active-bin count of the block
    uint32_t next = 32;    // the next attempt's lane; 32: no block
};
__device__ __forceinline__ double inverse_time_factor(InverseTimeTable& T, uint64_t attempted_before,
                                                      uint64_t active_bins, double current, int lane) {
    if (active_bins == 0) return current;
    if (T.next >= 32 || active_bins != T.active) {
        T.active = active_bins;
        T.next = 0;
        T.q = static_cast<double>(active_bins) /
              static_cast<double>(attempted_before + static_cast<uint64_t>(lane) + 1);
    }
    return __shfl_sync(kFull, T.q, static_cast<int>(T.next++));
}

// inverse_time_factor with a 32-bit count of active bins (a window has fewer than 2^31 bins)
// and the no-active-bin case as a select, so that the table refresh is the only branch of the
// per-attempt factor.
struct InverseTimeTable32 {
    double q = 0.0;         // lane j: active / (first + j + 1)
    uint32_t active = 0;    // active-bin count of the block
    uint32_t next = 32;     // the next attempt's lane; 32: no block
};
__device__ __forceinline__ double inverse_time_factor_select(InverseTimeTable32& T, uint64_t attempted_before,
                                                             uint32_t active_bins, double current, int lane) {
    if (T.next >= 32 || active_bins != T.active) {
        T.active = active_bins;
        T.next = 0;
        T.q = static_cast<double>(active_bins) /
              static_cast<double>(attempted_before + static_cast<uint64_t>(lane) + 1);
    }
    const double q = __shfl_sync(kFull, T.q, static_cast<int>(T.next++));
    return active_bins == 0 ? current : q;
}
// The same table with the refresh taken out of the per-attempt path: a caller that tests
// (T.next >= 32 || active_bins != T.active) in a branch of its own calls the refresh there,
// before the attempt, with the attempts made so far; the factor of the attempt is then a
// shuffle and a select.
__device__ __forceinline__ void inverse_time_refresh(InverseTimeTable32& T, uint64_t attempted_before,
                                                     uint32_t active_bins, int lane) {
    T.active = active_bins;
    T.next = 0;
    T.q = static_cast<double>(active_bins) / static_cast<double>(attempted_before + static_cast<uint64_t>(lane) + 1);
}
__device__ __forceinline__ double inverse_time_factor_next(InverseTimeTable32& T, uint32_t active_bins, double current) {
    const double q = __shfl_sync(kFull, T.q, static_cast<int>(T.next++));
    return active_bins == 0 ? current : q;
}

// Floor of a bin coordinate 0 <= q < 2^31 (the grid index of an in-range energy): the sum
// q + 2^52 rounded toward -infinity is 2^52 + floor(q) exactly (the unit in the last place is
// 1 there), and its low word is floor(q).  One add instead of a double-to-integer conversion.
__device__ __forceinline__ int bin_floor(double q) { return __double2loint(__dadd_rd(q, 0x1.0p52)); }

// update_round_trip_state (src/wang_landau.cpp:317-330)
__device__ __forceinline__ void round_trip_update(double energy, double lower, double upper, double margin_fraction,
                                                  int32_t& state, uint64_t& trips) {
    const double margin = margin_fraction * (upper - lower);
    if (energy <= lower + margin) {
        if (state == 2) {
            ++trips;
            state = 1;
        } else if (state == 0) {
            state = 1;
        }
    } else if (energy >= upper - margin && state == 1) {
        state = 2;
    }
}

// update_representatives (src/wang_landau.cpp:332-342); spins is the walker's current
// configuration (shared or global memory), n bytes, copied by the whole warp.
__device__ __forceinline__ void warp_update_representatives(const EngineView& v, int walker, double energy,
                                                            const int8_t* spins, int lane) {
    for (int r = 0; r < kRepresentatives; ++r) {
        const size_t q = static_cast<size_t>(walker) * kRepresentatives + r;
        const double distance = fabs(energy - v.rep_target[q]);
        if (distance < v.rep_dist[q]) {
            int8_t* dst = v.rep_spins + q * static_cast<size_t>(v.ld);
            for (int i = lane; i < v.ld; i += 32) dst[i] = spins[i];
            __syncwarp();
            if (lane == 0) {
                v.rep_dist[q] = distance;
                v.rep_energy[q] = energy;
                v.rep_present[q] = 1;
            }
            __syncwarp();
        }
    }
}

// ---- shared-memory carve-up of one walker --------------------------------------------

__host__ __device__ inline size_t round16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

struct SmemLayout {
    size_t fields, log_g, hist, sq, ds, spins, active, refine, total;
};

__host__ __device__ inline SmemLayout smem_layout(int ld, int mwb, bool smem_fields, bool features,
                                                  bool smem_spins = true) {
    SmemLayout L;
    size_t at = 0;
    L.fields = at; at += smem_fields ? static_cast<size_t>(ld) * 8 : 0;
    L.log_g = at; at += round16(static_cast<size_t>(mwb) * 8);
    L.hist = at; at += round16(static_cast<size_t>(mwb) * 8);
    L.sq = at; at += features ? round16(static_cast<size_t>(mwb) * 8) : 0;
    L.ds = at; at += features ? round16(static_cast<size_t>(mwb) * 8) : 0;
    L.spins = at; at += smem_spins ? round16(static_cast<size_t>(ld)) : 0;
    L.active = at; at += round16(static_cast<size_t>(mwb));
    L.refine = at; at += features ? round16(static_cast<size_t>(mwb)) : 0;
    L.total = at;
    return L;
}

__device__ __forceinline__ double window_lower(const EngineView& v, int wb) {
    return v.grid.minimum + static_cast<double>(wb) * v.grid.width;
}

__device__ __forceinline__ void record_error(Control* ctl, int status, int walker) {
    if (atomicCAS(&ctl->error, 0, status) == 0) ctl->error_walker = walker;
    ctl->done = 1;
}

}  // namespace wlg
