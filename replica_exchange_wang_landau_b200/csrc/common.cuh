// common.cuh — types and scalar helpers shared by the host engine and the sm_100a kernels.
//
// Every floating-point expression that the reference evaluates is evaluated here in the
// same order with IEEE double operations; the library is compiled with --fmad=false so
// that no multiply-add is contracted (the reference's ISO C++20 x86-64 build has none).
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#define WLG_HD __host__ __device__ __forceinline__

namespace wlg {

// ---- xoshiro256** with splitmix64 seeding (include/wl/rng.hpp:10-56) ---------------

WLG_HD uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

WLG_HD uint64_t splitmix_next(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s0, s1, s2, s3;

    // Xoshiro256StarStar(seed, stream): rng.hpp:52-55
    WLG_HD void seed(uint64_t seed_value, uint64_t stream) {
        uint64_t x = seed_value ^ (0xd2b74407b1ce6e93ULL * (stream + 1));
        s0 = splitmix_next(x);
        s1 = splitmix_next(x);
        s2 = splitmix_next(x);
        s3 = splitmix_next(x);
    }
    // operator(): rng.hpp:16-23
    WLG_HD uint64_t next() {
        const uint64_t result = rotl64(s1 * 5, 7) * 9;
        const uint64_t t = s1 << 17;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = rotl64(s3, 45);
        return result;
    }
};

// The inverse of Rng::next()'s state transition (the transition is an invertible linear map
// over GF(2)).  A sweep that generates draws ahead of their use rewinds its state by the
// number of unused draws, so the state it stores is the one after the consumed draws.
WLG_HD void rng_step_back(Rng& r) {
    // forward: a2 = s2^s0, a3 = s3^s1, a1 = s1^a2, a0 = s0^a3, b2 = a2^(s1<<17), b3 = rotl(a3,45)
    const uint64_t a3 = (r.s3 >> 45) | (r.s3 << 19);  // rotr(b3, 45)
    const uint64_t s0 = r.s0 ^ a3;
    // a1 ^ b2 = s1 ^ (s1 << 17); invert x ^ (x << 17)
    const uint64_t y = r.s1 ^ r.s2;
    const uint64_t s1 = y ^ (y << 17) ^ (y << 34) ^ (y << 51);
    const uint64_t a2 = r.s2 ^ (s1 << 17);
    r.s0 = s0;
    r.s1 = s1;
    r.s2 = a2 ^ s0;
    r.s3 = a3 ^ s1;
}

// uniform(): rng.hpp:25-27 — exact for the 53-bit integer.
WLG_HD double to_uniform(uint64_t x) { return static_cast<double>(x >> 11) * 0x1.0p-53; }

// x % bound for a bound fixed per system, without a 64-bit hardware divide: m =
// floor((2^64-1)/bound) underestimates the quotient by less than 2, so at most two
// corrections give the exact remainder (Barrett reduction).
struct FastMod {
    uint64_t bound;
    uint64_t m;
    uint64_t threshold;  // (-bound) % bound, the rejection threshold of bounded()
    uint64_t mask;       // bound - 1 when bound is a power of two (x % bound == x & mask)
    int32_t pow2;
    int32_t pad;
};

inline FastMod make_fastmod(uint64_t bound) {
    FastMod f;
    f.bound = bound;
    f.m = bound ? (~0ULL) / bound : 0;
    f.threshold = bound ? (0ULL - bound) % bound : 0;
    f.pow2 = bound != 0 && (bound & (bound - 1)) == 0;
    f.mask = bound ? bound - 1 : 0;
    f.pad = 0;
    return f;
}

WLG_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) >> 64);
#endif
}

WLG_HD uint64_t fast_mod(const FastMod& f, uint64_t x) {
    if (f.pow2) return x & f.mask;  // threshold is 0: no draw is ever rejected
    uint64_t r = x - mulhi64(x, f.m) * f.bound;
    if (r >= f.bound) r -= f.bound;
    if (r >= f.bound) r -= f.bound;
    return r;
}

// bounded(): rng.hpp:29-36 (bound > 0 here)
WLG_HD uint64_t bounded(Rng& rng, const FastMod& f) {
    for (;;) {
        const uint64_t x = rng.next();
        if (x >= f.threshold) return fast_mod(f, x);
    }
}

// ---- energy grid (src/wang_landau.cpp:13-38) -----------------------------------------

struct Grid {
    double minimum;
    double maximum;
    double width;
    int64_t count;       // llround((maximum - minimum) / width)
    double inv_width;    // 1 / width, exact when width is a power of two
    int32_t pow2_width;  // width is a power of two: x / width == x * inv_width exactly
    int32_t pad;
};

inline Grid make_grid(double minimum, double maximum, double width, int64_t count) {
    Grid g{minimum, maximum, width, count, 1.0 / width, 0, 0};
    int exponent = 0;
    g.pow2_width = std::frexp(width, &exponent) == 0.5 ? 1 : 0;
    return g;
}

// EnergyGrid::index; -1 for std::nullopt.  `!(e >= min && e <= max)` also rejects NaN
// and infinities, which is what `!isfinite(e) || e < min || e > max` does.  Dividing by a
// power-of-two width and multiplying by its (exact) reciprocal give the same rounded
// value, so the multiply is used whenever the width allows it.
WLG_HD int64_t grid_index(const Grid& g, double e) {
    if (!(e >= g.minimum && e <= g.maximum)) return -1;
    const double offset = e - g.minimum;
    const double q = g.pow2_width ? offset * g.inv_width : offset / g.width;
    uint64_t raw = static_cast<uint64_t>(floor(q));
    if (raw == static_cast<uint64_t>(g.count) && e == g.maximum) raw = static_cast<uint64_t>(g.count) - 1;
    if (raw >= static_cast<uint64_t>(g.count)) return -1;
    return static_cast<int64_t>(raw);
}

// ---- the histogram mean of histogram_statistics (src/wang_landau.cpp:349-361) --------
//
// The reference sums the histogram in long double (x87, 64-bit significand) and computes
// mean = (double)(total / (long double)active_bins): the quotient is rounded to 64
// significant bits and then to 53.  This restates that double rounding with integer
// arithmetic so that the device produces the same double.
WLG_HD double x87_mean(uint64_t total, uint64_t count) {
    if (total == 0 || count == 0) return 0.0;
    // Binary expansion of total/count: integer part q, then fraction bits from r.
    const uint64_t q = total / count;
    uint64_t r = total % count;
    // Collect 66 significant bits (64 kept + round bit + one more) and a sticky flag.
    uint64_t hi = 0;   // up to 64 significant bits
    int nbits = 0;     // significant bits collected into hi
    int exp2 = 0;      // value = hi * 2^exp2 (before rounding) ... tracked below
    int guard = 0, sticky = 0;
    // integer part
    int qbits = 0;
    for (uint64_t t = q; t; t >>= 1) ++qbits;
    if (qbits > 0) {
        if (qbits <= 64) { hi = q; nbits = qbits; exp2 = 0; }
    }
    // fraction bits (each step yields one bit of r/count)
    int frac_index = 0;  // number of fraction bits consumed
    while (nbits < 64) {
        r <<= 1;  // r < count <= 2^63 is required (count is a bin count)
        const int bit = r >= count ? 1 : 0;
        if (bit) r -= count;
        ++frac_index;
        if (nbits == 0 && !bit) continue;  // leading zeros of a value < 1
        hi = (hi << 1) | static_cast<uint64_t>(bit);
        ++nbits;
    }
    exp2 = -frac_index;
    // next bit = round bit for the 64-bit rounding; sticky = any remainder beyond
    {
        r <<= 1;
        guard = r >= count ? 1 : 0;
        if (guard) r -= count;
        sticky = r != 0 ? 1 : 0;
    }
    // round to 64 bits, nearest-even
    uint64_t m64 = hi;
    if (guard && (sticky || (m64 & 1))) {
        ++m64;
        if (m64 == 0) {  // carried out of 64 bits: 2^64
            m64 = 1ULL << 63;
            exp2 += 1;
        }
    }
    // value = m64 * 2^exp2 with m64 normalised (bit 63 set) — round to 53 bits, nearest-even
    const uint64_t low = m64 & 0x7FFULL;  // the 11 bits that are dropped
    uint64_t m53 = m64 >> 11;
    int e53 = exp2 + 11;
    if (low > 0x400ULL || (low == 0x400ULL && (m53 & 1))) {
        ++m53;
        if (m53 == (1ULL << 53)) {
            m53 >>= 1;
            e53 += 1;
        }
    }
    return ldexp(static_cast<double>(m53), e53);
}

// ---- device-side walker state -------------------------------------------------------

enum Stage : int32_t { kWangLandau = 0, kInverseTime = 1, kFrozen = 2 };

// Scalar state of one walker (the members of WangLandauWalker that change during a run,
// include/wl/wang_landau.hpp:141-168, plus run_rewl's last_flatness_check).
struct alignas(16) WalkerState {
    uint64_t rng[4];
    double energy;
    double factor;
    uint64_t attempted;
    uint64_t accepted;
    uint64_t forced;
    uint64_t last_accepted;
    uint64_t active_count;
    uint64_t refine_count;
    uint64_t last_check;
    uint64_t round_trips;
    double last_flatness;
    int32_t stage;
    int32_t cur_bin;       // grid_index(energy), -1 if none
    int32_t slot;          // configuration slot holding this walker's spins and fields
    int32_t window;        // window index
    int32_t rt_state;      // round-trip state machine
    int32_t rep_pending;   // representatives must be refreshed before the next batch
    // 1/t stage: attempts counted as made before this run, f = active / (attempted +
    // time_offset).  0 is the reference's rule.  A warm start that continues the schedule
    // (wlg_engine_warm_start_continue) sets kContinueSchedule; the first covered check then
    // enters the 1/t stage at the factor reached and sets the offset that makes the 1/t
    // factor start there.
    uint64_t time_offset;
};
constexpr uint64_t kContinueSchedule = ~0ULL;

// Run-wide control block written by the kernels and read by the host.
struct alignas(16) Control {
    uint64_t epoch;
    uint64_t exchange_attempted;
    uint64_t exchange_accepted;
    int32_t done;
    int32_t error;          // first wlg_status raised on the device (0 = none)
    int32_t error_walker;
    uint32_t frozen;        // walkers frozen after this epoch's check
    uint32_t at_limit;      // walkers at the attempt limit after this epoch's batch
    int32_t pad[3];
};

// Accumulated by the periodic FP64 recompute of a mixed-precision run (precision.cu).
struct PrecisionReport {
    unsigned long long max_field_drift_bits;   // max |h - h64| (bits of a non-negative double)
    unsigned long long max_energy_drift_bits;  // max |E - E64|
    unsigned long long recomputes;             // recompute passes applied
    unsigned long long resynced;               // walker resyncs applied
    unsigned long long deferred;               // resyncs deferred: E64 outside the window
    unsigned long long bin_changes;            // resyncs that moved the current bin
    unsigned long long pad[2];
};

struct DeviceParams {  // wl::WlParameters + the run_rewl intervals, on the device
    double flatness;
    uint64_t minimum_visits;
    double final_factor;
    uint64_t check_interval;  // max(1, check_interval_attempts)
    uint64_t force_after;
    int32_t inverse_time;
    int32_t nalivaiko;
    int32_t collect;
    int32_t withhold_draws;  // failure injection: producers publish no draws (wlg_engine_inject_wait_timeout)
    double round_trip_margin;
    uint64_t exchange_interval;
    uint64_t max_attempts;     // 0 = unlimited
    uint64_t seed;
};

constexpr int kRepresentatives = 9;

// Everything a kernel needs, passed by value.
struct EngineView {
    int32_t n;            // spins
    int32_t ld;           // padded row stride of J, spins and fields (multiple of 16)
    FastMod site_mod;     // bounded(n)
    int32_t precision;    // wlg_precision
    int32_t csr;
    const double* J64;             // dense ld x ld (rows padded with zeros)
    const float* J32;
    const __nv_bfloat16* J16;
    const float* Jscale;           // per-row scale of J16
    const int32_t* csr_ptr;        // n + 1
    const int32_t* csr_col;
    const double* csr_val64;
    const float* csr_val32;
    const int32_t* ell_col;        // ELLPACK copy of the CSR rows: n x ell_width, column -1 pads
    const double* ell_val64;       // FP64 couplings (FP64 runs)
    const float* ell_val32;        // FP32 couplings (FP32 runs)
    int32_t ell_width;             // 32, 64, 128 or 256; 0 when not built
    int32_t spins_global;          // the generic sweep and the initialisation read spins from HBM
    int32_t split_ring_log;        // split sweep: log2 of its draw / J-row staging ring (4 or 5; 0 = 4)
    Grid grid;
    int32_t walkers;
    int32_t walkers_per_window;
    int32_t windows;
    int32_t max_window_bins;
    const int32_t* win_begin;      // per window
    const int32_t* win_end;
    WalkerState* ws;
    double* log_g;                 // walkers x bins
    uint64_t* hist;                // walkers x bins
    uint8_t* active;               // walkers x bins
    uint8_t* refine;               // walkers x bins (Nalivaiko)
    double* sqdisp;                // walkers x bins (adaptive pilot)
    uint64_t* dsamples;            // walkers x bins
    int8_t* spins;                 // slots x ld
    double* fields;                // slots x ld
    double* rep_energy;            // walkers x 9
    double* rep_dist;              // walkers x 9
    double* rep_target;            // walkers x 9
    uint8_t* rep_present;          // walkers x 9
    int8_t* rep_spins;             // walkers x 9 x ld
    DeviceParams p;
    Control* ctl;
};

}  // namespace wlg
