// walker.cu — the walker kernels: target-Metropolis initialisation and the REWL sweep.
//
// walk_kernel is the hot path: WangLandauWalker::run_attempts / attempt_flip
// (src/wang_landau.cpp:244-315) for a batch of exchange_interval attempts, followed by the
// walker-local flatness / 1/t check of run_rewl (src/parallel.cpp:395-407).  One warp owns
// one walker for the whole batch; its local fields, spins and the window slice of
// log_g / H / active live in shared memory.  On an accepted flip the warp streams the J
// row of the flipped site (equal to the column the reference reads, because both triangles
// of J hold the same doubles, src/physics.cpp:180-181) with 16-byte coalesced read-only
// loads and updates the N fields in shared memory; the CSR form updates the z neighbours.
//
// init_kernel is the WangLandauWalker constructor (src/wang_landau.cpp:63-242).
#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

// ---- field updates: fields[j] += m * J[i][j]  (add_flip_delta, src/physics.cpp:190-236) ----
//
// m = -2 * old_spin is +-2, so m * J is exact and fma(m, J, h) rounds the same real number
// h + m*J once, exactly like the reference's separate multiply and add.

template <int kPrec>
__device__ __forceinline__ void dense_update(const EngineView& v, int i, double m, double* __restrict__ f,
                                             int lane) {
    if constexpr (kPrec == WLG_PRECISION_FP64) {
        const double2* __restrict__ row = reinterpret_cast<const double2*>(v.J64 + static_cast<size_t>(i) * v.ld);
        double2* f2 = reinterpret_cast<double2*>(f);
        const int n2 = v.ld >> 1;
        int k = lane;
        for (; k + 32 * 7 < n2; k += 32 * 8) {
            double2 a[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = __ldg(row + k + 32 * u);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                double2 h = f2[k + 32 * u];
                h.x = fma(m, a[u].x, h.x);
                h.y = fma(m, a[u].y, h.y);
                f2[k + 32 * u] = h;
            }
        }
        for (; k < n2; k += 32) {
            const double2 a = __ldg(row + k);
            double2 h = f2[k];
            h.x = fma(m, a.x, h.x);
            h.y = fma(m, a.y, h.y);
            f2[k] = h;
        }
    } else if constexpr (kPrec == WLG_PRECISION_FP32) {
        const float4* __restrict__ row = reinterpret_cast<const float4*>(v.J32 + static_cast<size_t>(i) * v.ld);
        double2* f2 = reinterpret_cast<double2*>(f);
        const int n4 = v.ld >> 2;
        for (int k = lane; k < n4; k += 32) {
            const float4 a = __ldg(row + k);
            double2 h0 = f2[2 * k], h1 = f2[2 * k + 1];
            h0.x = fma(m, static_cast<double>(a.x), h0.x);
            h0.y = fma(m, static_cast<double>(a.y), h0.y);
            h1.x = fma(m, static_cast<double>(a.z), h1.x);
            h1.y = fma(m, static_cast<double>(a.w), h1.y);
            f2[2 * k] = h0;
            f2[2 * k + 1] = h1;
        }
    } else {
        const uint4* __restrict__ row = reinterpret_cast<const uint4*>(v.J16 + static_cast<size_t>(i) * v.ld);
        const double ms = m * static_cast<double>(v.Jscale[i]);
        double2* f2 = reinterpret_cast<double2*>(f);
        const int n8 = v.ld >> 3;
        for (int k = lane; k < n8; k += 32) {
            const uint4 raw = __ldg(row + k);
            const uint32_t words[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float lo = __uint_as_float(words[q] << 16);
                const float hi = __uint_as_float(words[q] & 0xffff0000u);
                double2 h = f2[4 * k + q];
                h.x = fma(ms, static_cast<double>(lo), h.x);
                h.y = fma(ms, static_cast<double>(hi), h.y);
                f2[4 * k + q] = h;
            }
        }
    }
}

template <int kPrec>
__device__ __forceinline__ void csr_update(const EngineView& v, int i, double m, double* f, int lane) {
    const int begin = v.csr_ptr[i], end = v.csr_ptr[i + 1];
    for (int k = begin + lane; k < end; k += 32) {
        const int c = __ldg(v.csr_col + k);
        const double val = kPrec == WLG_PRECISION_FP64 ? __ldg(v.csr_val64 + k) : static_cast<double>(__ldg(v.csr_val32 + k));
        f[c] = fma(m, val, f[c]);
    }
}

template <int kPrec, bool kCsr>
__device__ __forceinline__ void flip_update(const EngineView& v, int i, double m, double* f, int lane) {
    if constexpr (kCsr) csr_update<kPrec>(v, i, m, f, lane);
    else dense_update<kPrec>(v, i, m, f, lane);
}

// local_fields (src/physics.cpp:238-251) by one warp: lanes over sites, each site summed
// sequentially over j in the reference's order (always from the FP64 couplings).
template <bool kCsr>
__device__ void warp_local_fields(const EngineView& v, const int8_t* s, double* f, int lane) {
    if constexpr (!kCsr) {
        for (int base = 0; base < v.n; base += 256) {
            double acc[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = 0.0;
            for (int j = 0; j < v.n; ++j) {
                const double sj = static_cast<double>(s[j]);
                const double* row = v.J64 + static_cast<size_t>(j) * v.ld + base + lane;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (base + lane + 32 * c < v.n) acc[c] += row[32 * c] * sj;
            }
#pragma unroll
            for (int c = 0; c < 8; ++c)
                if (base + lane + 32 * c < v.n) f[base + lane + 32 * c] = acc[c];
        }
    } else {
        for (int i = lane; i < v.n; i += 32) {
            double sum = 0.0;
            for (int q = v.csr_ptr[i]; q < v.csr_ptr[i + 1]; ++q) sum += v.csr_val64[q] * static_cast<double>(s[v.csr_col[q]]);
            f[i] = sum;
        }
    }
    __syncwarp();
}

// total_energy (src/physics.cpp:253-259): lane 0 sums sequentially, result broadcast.
__device__ __forceinline__ double warp_total_energy(const EngineView& v, const int8_t* s, const double* f, int lane) {
    double e = 0.0;
    if (lane == 0)
        for (int i = 0; i < v.n; ++i) e += 0.5 * static_cast<double>(s[i]) * f[i];
    return __shfl_sync(kFull, e, 0);
}

// ---- shared-memory carve-up ---------------------------------------------------------------

size_t walker_smem_bytes(const EngineView& v, bool smem_fields, bool features) {
    return smem_layout(v.ld, v.max_window_bins, smem_fields, features, v.spins_global == 0).total;
}

bool fields_fit_in_smem(const EngineView& v, bool features) {
    return walker_smem_bytes(v, true, features) <= 200 * 1024;
}

// ---- the sweep -----------------------------------------------------------------------------

template <int kPrec, bool kCsr, bool kSmemF, bool kFeat>
__global__ void __launch_bounds__(256) walk_kernel(EngineView v, WalkArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int local = blockIdx.x * (blockDim.x >> 5) + warp;
    if (local >= a.count) return;
    const int w = a.first + local;
    Control* ctl = v.ctl;
    if (a.epoch_mode && *reinterpret_cast<volatile int32_t*>(&ctl->done)) return;

    const SmemLayout L = smem_layout(v.ld, v.max_window_bins, kSmemF, kFeat, v.spins_global == 0);
    unsigned char* base = smem + static_cast<size_t>(warp) * a.smem_per_walker;
    double* lg_s = reinterpret_cast<double*>(base + L.log_g);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(base + L.hist);
    double* sq_s = reinterpret_cast<double*>(base + L.sq);
    uint64_t* ds_s = reinterpret_cast<uint64_t*>(base + L.ds);
    uint8_t* act_s = base + L.active;
    uint8_t* ref_s = base + L.refine;

    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    const size_t boff = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + static_cast<size_t>(wb);
    double* fg = v.fields + static_cast<size_t>(st.slot) * v.ld;
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * v.ld;
    int8_t* sp_s = v.spins_global ? sg : reinterpret_cast<int8_t*>(base + L.spins);
    double* f = kSmemF ? reinterpret_cast<double*>(base + L.fields) : fg;
    const DeviceParams& P = v.p;
    const bool collect = kFeat && P.collect;
    const bool nalivaiko = kFeat && P.nalivaiko;

    // stage the walker into shared memory
    if constexpr (kSmemF) {
        const double2* src = reinterpret_cast<const double2*>(fg);
        double2* dst = reinterpret_cast<double2*>(f);
        for (int k = lane; k < (v.ld >> 1); k += 32) dst[k] = src[k];
    }
    if (!v.spins_global) {
        const int4* src = reinterpret_cast<const int4*>(sg);
        int4* dst = reinterpret_cast<int4*>(sp_s);
        for (int k = lane; k < (v.ld >> 4); k += 32) dst[k] = src[k];
    }
    for (int b = lane; b < nbins; b += 32) {
        lg_s[b] = v.log_g[boff + b];
        h_s[b] = v.hist[boff + b];
        act_s[b] = v.active[boff + b];
        if constexpr (kFeat) {
            ref_s[b] = v.refine[boff + b];
            if (collect) {  // the pilot arrays exist only in pilot runs
                sq_s[b] = v.sqdisp[boff + b];
                ds_s[b] = v.dsamples[boff + b];
            }
        }
    }
    __syncwarp();

    if (collect && st.rep_pending) {  // a replica exchange changed the configuration
        warp_update_representatives(v, w, st.energy, sp_s, lane);
        st.rep_pending = 0;
    }

    int cur = st.cur_bin;
    if (cur < wb || cur >= we) {  // "Walker escaped its energy window"
        if (lane == 0) record_error(ctl, WLG_ERR_ESCAPED, w);
        return;
    }

    uint64_t batch;
    if (a.fixed_batch) {
        batch = a.fixed_batch;
    } else {
        batch = P.exchange_interval;
        if (P.max_attempts) {
            const uint64_t remaining = st.attempted < P.max_attempts ? P.max_attempts - st.attempted : 0;
            batch = remaining < batch ? remaining : batch;
        }
    }

    Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};
    double E = st.energy;
    double factor = st.factor;
    int32_t stage = st.stage;
    uint64_t att = st.attempted, acc_n = st.accepted, forced_n = st.forced, last_acc = st.last_accepted;
    uint64_t active_count = st.active_count, refine_count = st.refine_count;
    int32_t rt_state = st.rt_state;
    uint64_t trips = st.round_trips;
    const double lower = window_lower(v, wb);
    const double upper = window_lower(v, we);

    // the current bin lives in registers
    double lg_cur = lg_s[cur - wb];
    uint64_t hc_cur = h_s[cur - wb];
    bool act_cur = act_s[cur - wb] != 0;
    bool ref_cur = nalivaiko ? ref_s[cur - wb] != 0 : true;

    for (uint64_t t = 0; t < batch; ++t) {
        const int i = static_cast<int>(bounded(rng, v.site_mod));
        const int8_t si = sp_s[i];
        const double delta = -2.0 * static_cast<double>(si) * f[i];
        const double Ep = E + delta;
        const int64_t nb = grid_index(v.grid, Ep);
        bool accepted = false, forced = false;
        double lg_new = 0.0;
        if (nb >= wb && nb < we) {
            lg_new = nb == cur ? lg_cur : lg_s[nb - wb];
            const double log_ratio = lg_cur - lg_new;
            const bool force_due = P.force_after != 0 && att - last_acc >= P.force_after;
            if (log_ratio >= 0.0) {
                accepted = true;
            } else if (force_due) {
                accepted = forced = true;
            } else {
                const double u = to_uniform(rng.next());
                accepted = log_uniform_below(u, log_ratio);
            }
        }
        ++att;
        if (accepted) {
            flip_update<kPrec, kCsr>(v, i, -2.0 * static_cast<double>(si), f, lane);
            if (lane == 0) sp_s[i] = static_cast<int8_t>(-si);
            E = Ep;
            ++acc_n;
            if (forced) ++forced_n;
            last_acc = att;
        }
        if (collect && lane == 0) {
            const double displacement = accepted ? delta : 0.0;
            sq_s[cur - wb] += displacement * displacement;
            ++ds_s[cur - wb];
        }
        if (stage == kInverseTime) {  // update_inverse_time_factor
            if (active_count != 0 && att != 0)
                factor = static_cast<double>(active_count) / static_cast<double>(att + st.time_offset);
            if (factor <= P.final_factor) stage = kFrozen;
        }
        // update_current_bin
        if (accepted && nb != cur) {
            if (lane == 0) {
                lg_s[cur - wb] = lg_cur;
                h_s[cur - wb] = hc_cur;
                act_s[cur - wb] = act_cur ? 1 : 0;
                if (nalivaiko) ref_s[cur - wb] = ref_cur ? 1 : 0;
            }
            cur = static_cast<int>(nb);
            lg_cur = lg_new;
            hc_cur = h_s[cur - wb];
            act_cur = act_s[cur - wb] != 0;
            ref_cur = nalivaiko ? ref_s[cur - wb] != 0 : true;
        }
        ++hc_cur;
        if (!act_cur) {
            act_cur = true;
            ++active_count;
        }
        if (nalivaiko && !ref_cur) {
            ref_cur = true;
            ++refine_count;
        }
        if (stage != kFrozen) lg_cur += factor;
        __syncwarp();
        if (collect && accepted) {
            round_trip_update(E, lower, upper, P.round_trip_margin, rt_state, trips);
            warp_update_representatives(v, w, E, sp_s, lane);
        }
    }
    // flush the register-held bin
    if (lane == 0) {
        lg_s[cur - wb] = lg_cur;
        h_s[cur - wb] = hc_cur;
        act_s[cur - wb] = act_cur ? 1 : 0;
        if (nalivaiko) ref_s[cur - wb] = ref_cur ? 1 : 0;
    }
    __syncwarp();

    st.rng[0] = rng.s0; st.rng[1] = rng.s1; st.rng[2] = rng.s2; st.rng[3] = rng.s3;
    st.energy = E;
    st.factor = factor;
    st.stage = stage;
    st.attempted = att;
    st.accepted = acc_n;
    st.forced = forced_n;
    st.last_accepted = last_acc;
    st.active_count = active_count;
    st.refine_count = refine_count;
    st.cur_bin = cur;
    st.rt_state = rt_state;
    st.round_trips = trips;

    // the walker-local check of run_rewl (src/parallel.cpp:395-407)
    if (a.epoch_mode && st.stage == kWangLandau) {
        const bool at_limit = P.max_attempts != 0 && st.attempted >= P.max_attempts;
        if (st.attempted - st.last_check >= P.check_interval || at_limit) {
            st.last_check = st.attempted;
            const HistStats hs = warp_histogram_statistics(h_s, nalivaiko ? ref_s : act_s, nbins,
                                                           nalivaiko ? st.refine_count : st.active_count, lane);
            st.last_flatness = P.inverse_time ? hs.coverage : hs.min_over_mean;
            if (stats_ready(hs, st.stage, P)) warp_begin_next_iteration(st, h_s, ref_s, nbins, P, lane);
        }
    }

    // write back
    if constexpr (kSmemF) {
        const double2* src = reinterpret_cast<const double2*>(f);
        double2* dst = reinterpret_cast<double2*>(fg);
        for (int k = lane; k < (v.ld >> 1); k += 32) dst[k] = src[k];
    }
    if (!v.spins_global) {
        const int4* src = reinterpret_cast<const int4*>(sp_s);
        int4* dst = reinterpret_cast<int4*>(sg);
        for (int k = lane; k < (v.ld >> 4); k += 32) dst[k] = src[k];
    }
    for (int b = lane; b < nbins; b += 32) {
        v.log_g[boff + b] = lg_s[b];
        v.hist[boff + b] = h_s[b];
        v.active[boff + b] = act_s[b];
        if constexpr (kFeat) {
            v.refine[boff + b] = ref_s[b];
            if (collect) {
                v.sqdisp[boff + b] = sq_s[b];
                v.dsamples[boff + b] = ds_s[b];
            }
        }
    }
    if (lane == 0) {
        v.ws[w] = st;
        if (a.epoch_mode) {
            if (st.stage == kFrozen) atomicAdd(&ctl->frozen, 1u);
            if (P.max_attempts != 0 && st.attempted >= P.max_attempts) atomicAdd(&ctl->at_limit, 1u);
        }
    }
}

// ---- initialisation: the WangLandauWalker constructor --------------------------------------

template <int kPrec, bool kCsr, bool kSmemF, bool kFeat>
__global__ void __launch_bounds__(256) init_kernel(EngineView v, InitArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int w = blockIdx.x * (blockDim.x >> 5) + warp;
    if (w >= v.walkers) return;

    const SmemLayout L = smem_layout(v.ld, v.max_window_bins, kSmemF, kFeat, v.spins_global == 0);
    unsigned char* base = smem + static_cast<size_t>(warp) * a.smem_per_walker;
    double* fg = v.fields + static_cast<size_t>(w) * v.ld;
    int8_t* sg = v.spins + static_cast<size_t>(w) * v.ld;
    int8_t* s = v.spins_global ? sg : reinterpret_cast<int8_t*>(base + L.spins);
    double* f = kSmemF ? reinterpret_cast<double*>(base + L.fields) : fg;

    WalkerState st = v.ws[w];  // window, slot and zeroed counters prepared by the host
    const int wb = v.win_begin[st.window], we = v.win_end[st.window];
    const bool supplied = a.initial_spins != nullptr && a.present[w] != 0;
    for (int i = lane; i < v.ld; i += 32)
        s[i] = i < v.n ? (supplied ? a.initial_spins[static_cast<size_t>(w) * v.ld + i] : static_cast<int8_t>(1)) : 0;
    if constexpr (kSmemF)
        for (int i = lane; i < v.ld; i += 32) f[i] = 0.0;
    __syncwarp();
    warp_local_fields<kCsr>(v, s, f, lane);
    double E = warp_total_energy(v, s, f, lane);

    Rng rng;
    rng.seed(v.p.seed, static_cast<uint64_t>(w));
    const Grid& g = v.grid;
    auto in_window = [&](int64_t b) { return b >= wb && b < we; };

    InitReport rep{};
    bool ok = false;
    if (supplied && in_window(grid_index(g, E))) {
        ok = true;
    } else {
        const double lower = g.minimum + static_cast<double>(wb) * g.width;
        const double upper = g.minimum + static_cast<double>(we) * g.width;
        const double span = upper - lower;
        const double target = 0.5 * (lower + upper);
        const double target_fraction = supplied ? 1.0 : a.target_fraction;
        const double half = 0.5 * target_fraction * span;
        const double tf_span = a.temperature_fraction * span;
        const double T0 = g.width < tf_span ? tf_span : g.width;                    // std::max
        const double mt_span = a.max_temperature_fraction * span;
        const double Tmax = T0 < mt_span ? mt_span : T0;                            // std::max
        double T = T0;
        const uint64_t n = static_cast<uint64_t>(v.n);
        const uint64_t stall = a.stall_per_spin > (~0ULL) / n ? ~0ULL : a.stall_per_spin * n;
        uint64_t since = 0, increases = 0, restarts = 0;
        double highest = T;
        double min_r = E, max_r = E, closest = E, cdist = fabs(E - target);
        auto record = [&](double c) {
            min_r = c < min_r ? c : min_r;
            max_r = max_r < c ? c : max_r;
            const double d = fabs(c - target);
            if (d < cdist) {
                cdist = d;
                closest = c;
                return true;
            }
            return false;
        };
        auto in_band = [&](double e) { return in_window(grid_index(g, e)) && fabs(e - target) <= half; };
        for (uint64_t step = 0; step < a.init_max_attempts; ++step) {
            if (in_band(E)) { ok = true; break; }
            if (since >= stall) {
                if (T < Tmax) {
                    const double raised = T * a.temperature_multiplier;
                    T = raised < Tmax ? raised : Tmax;                              // std::min
                    highest = highest < T ? T : highest;                            // std::max
                    ++increases;
                } else {
                    for (int i = 0; i < v.n; ++i) {  // bounded(2) per spin, in order
                        const uint64_t x = rng.next();
                        if (lane == (i & 31)) s[i] = (x & 1ULL) == 0 ? static_cast<int8_t>(-1) : static_cast<int8_t>(1);
                    }
                    __syncwarp();
                    warp_local_fields<kCsr>(v, s, f, lane);
                    E = warp_total_energy(v, s, f, lane);
                    record(E);
                    T = T0;
                    ++restarts;
                }
                since = 0;
                if (in_band(E)) { ok = true; break; }
            }
            const int i = static_cast<int>(bounded(rng, v.site_mod));
            const int8_t old = s[i];
            const double delta = -2.0 * static_cast<double>(old) * f[i];
            const double proposed = E + delta;
            const double log_acceptance = (fabs(E - target) - fabs(proposed - target)) / T;
            bool improved = false;
            if (log_acceptance >= 0.0 || log_uniform_below(to_uniform(rng.next()), log_acceptance)) {
                flip_update<WLG_PRECISION_FP64, kCsr>(v, i, -2.0 * static_cast<double>(old), f, lane);
                if (lane == 0) s[i] = static_cast<int8_t>(-old);
                E = proposed;
                improved = record(E);
            }
            __syncwarp();
            if (improved) since = 0;
            else if (since < ~0ULL) ++since;
        }
        if (!ok && in_band(E)) ok = true;
        rep.target = target;
        rep.half_width = half;
        rep.minimum_reached = min_r;
        rep.maximum_reached = max_r;
        rep.closest = closest;
        rep.closest_distance = cdist;
        rep.highest_temperature = highest;
        rep.increases = increases;
        rep.restarts = restarts;
        rep.stall = stall;
    }
    rep.status = ok ? 0 : 1;
    if (lane == 0) a.reports[w] = rep;
    if (!ok) return;

    // update_current_bin + update_round_trip_state + update_representatives
    const int64_t b = grid_index(g, E);
    const size_t at = static_cast<size_t>(w) * static_cast<size_t>(g.count) + static_cast<size_t>(b);
    st.energy = E;
    st.cur_bin = static_cast<int32_t>(b);
    st.rng[0] = rng.s0; st.rng[1] = rng.s1; st.rng[2] = rng.s2; st.rng[3] = rng.s3;
    st.factor = 1.0;
    st.stage = kWangLandau;
    st.active_count = 1;
    st.refine_count = v.p.nalivaiko ? 1 : 0;
    if (lane == 0) {
        v.hist[at] = 1;
        v.active[at] = 1;
        if (v.p.nalivaiko) v.refine[at] = 1;
        v.log_g[at] = 0.0 + 1.0;
    }
    if (kFeat && v.p.collect) {
        round_trip_update(E, window_lower(v, wb), window_lower(v, we), v.p.round_trip_margin, st.rt_state,
                          st.round_trips);
        warp_update_representatives(v, w, E, s, lane);
    }
    if constexpr (kSmemF)
        for (int i = lane; i < v.ld; i += 32) fg[i] = f[i];
    if (!v.spins_global)
        for (int i = lane; i < v.ld; i += 32) sg[i] = s[i];
    if (lane == 0) v.ws[w] = st;
}

// ---- dispatch ------------------------------------------------------------------------------

using WalkFn = void (*)(EngineView, WalkArgs);
using InitFn = void (*)(EngineView, InitArgs);

template <int P, bool C, bool S, bool F>
static void set_smem_attr(const void* fn) {
    static bool done = false;
    if (!done) {
        check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        done = true;
    }
}

template <int P, bool C, bool S, bool F>
static WalkFn walk_fn() {
    set_smem_attr<P, C, S, F>(reinterpret_cast<const void*>(&walk_kernel<P, C, S, F>));
    return &walk_kernel<P, C, S, F>;
}
template <int P, bool C, bool S, bool F>
static InitFn init_fn() {
    set_smem_attr<P + 8, C, S, F>(reinterpret_cast<const void*>(&init_kernel<P, C, S, F>));
    return &init_kernel<P, C, S, F>;
}

#define WLG_SELECT(GET, P, C)                                                    \
    if (smem_fields && features) return GET<P, C, true, true>();                \
    if (smem_fields && !features) return GET<P, C, true, false>();              \
    if (!smem_fields && features) return GET<P, C, false, true>();              \
    return GET<P, C, false, false>();

static WalkFn pick_walk(int precision, bool csr, bool smem_fields, bool features) {
    if (csr) {
        if (precision == WLG_PRECISION_FP32) { WLG_SELECT(walk_fn, WLG_PRECISION_FP32, true) }
        WLG_SELECT(walk_fn, WLG_PRECISION_FP64, true)
    }
    if (!smem_fields) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "dense couplings need the fields in shared memory");
    if (precision == WLG_PRECISION_FP32) {
        if (features) return walk_fn<WLG_PRECISION_FP32, false, true, true>();
        return walk_fn<WLG_PRECISION_FP32, false, true, false>();
    }
    if (precision == WLG_PRECISION_BF16) {
        if (features) return walk_fn<WLG_PRECISION_BF16, false, true, true>();
        return walk_fn<WLG_PRECISION_BF16, false, true, false>();
    }
    if (features) return walk_fn<WLG_PRECISION_FP64, false, true, true>();
    return walk_fn<WLG_PRECISION_FP64, false, true, false>();
}

static InitFn pick_init(bool csr, bool smem_fields, bool features) {
    if (csr) { WLG_SELECT(init_fn, WLG_PRECISION_FP64, true) }
    if (features) return init_fn<WLG_PRECISION_FP64, false, true, true>();
    return init_fn<WLG_PRECISION_FP64, false, true, false>();
}
#undef WLG_SELECT

static bool features_of(const EngineView& v) { return v.p.collect || v.p.nalivaiko; }

void launch_walk(const EngineView& v, const WalkArgs& a, int wpb, cudaStream_t stream) {
    const bool features = features_of(v);
    if (!v.csr && launch_sweep_dense(v, a, stream)) return;  // sweep.cu: the TMA row ring
    if (v.csr && launch_sweep_csr(v, a, wpb, stream)) return;  // sweep_csr.cu: ELLPACK rows, fields in HBM
    const bool smem_fields = a.smem_per_walker >= static_cast<int>(walker_smem_bytes(v, true, features));
    WalkFn fn = pick_walk(v.precision, v.csr != 0, smem_fields, features);
    wpb = std::max(1, std::min(wpb, 8));
    while (wpb > 1 && static_cast<size_t>(a.smem_per_walker) * wpb > 227 * 1024) --wpb;
    if (static_cast<size_t>(a.smem_per_walker) > 227 * 1024)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "walker state does not fit in shared memory");
    const unsigned blocks = static_cast<unsigned>((a.count + wpb - 1) / wpb);
    fn<<<blocks, 32 * wpb, static_cast<size_t>(a.smem_per_walker) * wpb, stream>>>(v, a);
    check_cuda(cudaGetLastError(), "walk_kernel");
}

void launch_init(const EngineView& v, const InitArgs& a, int wpb, cudaStream_t stream) {
    const bool features = features_of(v);
    const bool smem_fields = a.smem_per_walker >= static_cast<int>(walker_smem_bytes(v, true, features));
    InitFn fn = pick_init(v.csr != 0, smem_fields, features);
    wpb = std::max(1, std::min(wpb, 8));
    while (wpb > 1 && static_cast<size_t>(a.smem_per_walker) * wpb > 227 * 1024) --wpb;
    if (static_cast<size_t>(a.smem_per_walker) > 227 * 1024)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "walker state does not fit in shared memory");
    const unsigned blocks = static_cast<unsigned>((v.walkers + wpb - 1) / wpb);
    fn<<<blocks, 32 * wpb, static_cast<size_t>(a.smem_per_walker) * wpb, stream>>>(v, a);
    check_cuda(cudaGetLastError(), "init_kernel");
}

}  // namespace wlg
