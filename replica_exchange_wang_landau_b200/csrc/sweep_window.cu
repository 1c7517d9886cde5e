// sweep_window.cu — whole epochs of a single-window run of a small dense system in one launch:
// run_rewl's epoch loop (src/parallel.cpp:276-534) when there is one energy window, so no
// replica exchange happens, with each walker's batch of exchange_interval attempts
// (WangLandauWalker::run_attempts / attempt_flip, src/wang_landau.cpp:244-315) and its
// flatness / 1/t check (src/parallel.cpp:395-407) between epochs.
//
// The per-epoch launches of the other sweeps (a kernel node for the walk and one for the
// exchange, each staging the walker state in and out) cost a few microseconds, which is
// most of an epoch when a system has a handful of spins and the exchange interval is tens
// of attempts.  Here one CTA holds every walker of the window for many epochs:
//
// * Warp w < W is walker w's decision warp, warp W + w its draw producer (W walkers).
// * N <= 32: lane j keeps the field of site j in a register and the spins are a 32-bit mask
//   held by every lane; J (N x N FP64, at most 8 KB) is staged in shared memory.  A flip
//   updates every field at once, f_j = fma(m_eff, J_ij, f_j) on lane j, with m_eff = 0 for a
//   rejected flip (exact: a field is never -0.0, as the sums start at +0.0).
// * The next attempt's site is draw hq+1 or, when this attempt consumes the acceptance
//   uniform, draw hq+2 (the lookahead of the dense split sweep): both candidates' fields are
//   read by shuffles before the decision, and the chosen one is brought up to date with one
//   fma after it, so the chain is field -> proposed energy -> bin -> log g -> accept ->
//   next field, with no memory access but the log g load.
// * The producer generates the walker's draws 32 at a time (every lane steps the generator,
//   lane j keeps draw j, with its site and log(max(u, 2^-53)), src/wang_landau.cpp:250, 261)
//   into a 64-entry shared-memory ring, published with release stores; the walker publishes
//   the draws it has consumed once per batch of 32.  The draw stream runs on across the epochs of the launch; at
//   the end the generator is stepped back over the draws not consumed (rng_step_back).
// * At the end of an epoch each walker folds its histogram deltas, runs the check, and the
//   walker warps meet at a named barrier (the producers never take part); walker 0 decides
//   termination (every walker frozen, or every walker at the attempt limit, or an error,
//   src/parallel.cpp:527-533) and counts the epoch, as the exchange kernel does per epoch.
// * Every wait on another warp is bounded: a walker that waits too long for draws records
//   WLG_ERR_TIMEOUT, still takes part in the epoch's barrier (so the others end the run at
//   that epoch) and does not write its state back.
// The decision arithmetic is that of the split sweep, operation for operation.
#include <type_traits>

#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

namespace {

constexpr int kWindowRing = 64;                    // draw records per walker: two batches of 32
constexpr uint32_t kWindowRingMask = kWindowRing - 1;
constexpr uint32_t kWindowWaitPolls = 1u << 22;    // walker polls for a draw batch
constexpr uint32_t kWindowProducerPolls = 1u << 24;  // producer polls for ring room
constexpr int kWindowMaxWalkers = 4;               // 64 x 4 threads per CTA

struct WindowLayout {
    size_t J, shared_ctl, walkers, lg, h, site, lnu, ctl, hd, act, per_walker, total;
};
// J (ld x ld), the CTA's control words, then one region per walker.
__host__ __device__ inline WindowLayout window_layout(int ld, int mwb, int walkers) {
    WindowLayout L;
    size_t at = 0;
    L.J = at; at += static_cast<size_t>(ld) * static_cast<size_t>(ld) * 8;
    L.shared_ctl = at; at += 64;
    L.walkers = at;
    size_t w = 0;
    L.lg = w; w += round16(static_cast<size_t>(mwb) * 8);
    L.h = w; w += round16(static_cast<size_t>(mwb) * 8);
    L.site = w; w += kWindowRing * 4;
    L.lnu = w; w += kWindowRing * 8;
    L.ctl = w; w += 64;  // consumed, produced, stop, producer timeout; rng[4] at +16
    L.hd = w; w += round16(static_cast<size_t>(mwb) * 4);
    L.act = w; w += round16(static_cast<size_t>(mwb));
    L.per_walker = round16(w);
    L.total = at + L.per_walker * static_cast<size_t>(walkers);
    return L;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void st_release_u32(uint32_t addr, uint32_t value) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(addr), "r"(value) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(uint32_t addr) {
    uint32_t value;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(value) : "r"(addr) : "memory");
    return value;
}
// Barrier 1 over the walker warps only (barrier 0 is __syncthreads).
__device__ __forceinline__ void walkers_barrier(int threads) {
    asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

template <bool kPow2>
__global__ void __launch_bounds__(64 * kWindowMaxWalkers, 1) sweep_window_kernel(EngineView v, uint32_t epochs) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int W = v.walkers;
    const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
    const int ld = v.ld, n = v.n;
    const WindowLayout TL = window_layout(ld, v.max_window_bins, W);
    double* J_s = reinterpret_cast<double*>(smem + TL.J);
    int32_t* sc = reinterpret_cast<int32_t*>(smem + TL.shared_ctl);  // done, frozen, at limit, error
    Control* ctl = v.ctl;
    const bool producer = warp >= W;
    const int w = producer ? warp - W : warp;
    unsigned char* wb_s = smem + TL.walkers + TL.per_walker * static_cast<size_t>(w);
    double* lg_s = reinterpret_cast<double*>(wb_s + TL.lg);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(wb_s + TL.h);
    int32_t* rec_site = reinterpret_cast<int32_t*>(wb_s + TL.site);
    double* rec_lnu = reinterpret_cast<double*>(wb_s + TL.lnu);
    uint32_t* wctl = reinterpret_cast<uint32_t*>(wb_s + TL.ctl);
    uint64_t* wrng = reinterpret_cast<uint64_t*>(wb_s + TL.ctl + 16);
    uint32_t* hd = reinterpret_cast<uint32_t*>(wb_s + TL.hd);
    uint8_t* act_s = wb_s + TL.act;
    const uint32_t consumed_addr = smem_u32(wctl), produced_addr = consumed_addr + 4, stop_addr = consumed_addr + 8;

    for (int k = static_cast<int>(threadIdx.x); k < ld * ld; k += static_cast<int>(blockDim.x)) J_s[k] = v.J64[k];
    if (threadIdx.x == 0) {
        sc[0] = *reinterpret_cast<volatile int32_t*>(&ctl->done);
        sc[1] = 0;
        sc[2] = 0;
        sc[3] = 0;
    }
    if (producer && lane == 0) {
        wctl[0] = 0;
        wctl[1] = 0;
        wctl[2] = 0;
        wctl[3] = 0;
    }
    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    const size_t boff = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + static_cast<size_t>(wb);
    if (!producer) {
        for (int b = lane; b < nbins; b += 32) {
            lg_s[b] = v.log_g[boff + b];
            h_s[b] = v.hist[boff + b];
            act_s[b] = v.active[boff + b];
            hd[b] = 0;
        }
    }
    __syncthreads();
    if (sc[0]) return;  // the run has already terminated (every thread reads the same word)

    if (producer) {
        // ---- the walker's draws, 32 per batch, at most kWindowRing ahead of the walker ----
        const FastMod fm = v.site_mod;
        Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};
        uint32_t produced = 0, timeout = 0;
        // withhold_draws: publish nothing, so that the walkers' bounded waits run out
        for (bool open = v.p.withhold_draws == 0; open;) {
            uint32_t go = 0;
            if (lane == 0) {
                for (uint32_t polls = 0; polls < kWindowProducerPolls; ++polls) {
                    if (ld_acquire_u32(stop_addr)) break;
                    if (produced + 32 - ld_acquire_u32(consumed_addr) <= static_cast<uint32_t>(kWindowRing)) {
                        go = 1;
                        break;
                    }
                }
                if (!go && !ld_acquire_u32(stop_addr)) timeout = 1;
            }
            if (!__shfl_sync(kFull, go, 0)) break;
            __syncwarp();  // lane 0's acquire orders the walker's reads before this batch's writes
            uint64_t mine = 0;
#pragma unroll 4
            for (int j = 0; j < 32; ++j) {
                const uint64_t d = rng.next();
                mine = lane == j ? d : mine;
            }
            const uint32_t e = (produced + static_cast<uint32_t>(lane)) & kWindowRingMask;
            rec_site[e] = mine < fm.threshold ? -1 : static_cast<int>(fast_mod(fm, mine));
            rec_lnu[e] = log(fmax(to_uniform(mine), 0x1.0p-53));
            __syncwarp();
            produced += 32;
            if (lane == 0) st_release_u32(produced_addr, produced);
        }
        if (lane == 0) {
            wctl[3] = timeout;
            wrng[0] = rng.s0;
            wrng[1] = rng.s1;
            wrng[2] = rng.s2;
            wrng[3] = rng.s3;
        }
        __syncthreads();
        return;
    }

    // ---- walker w ----
    bool failed = false;
    if (st.cur_bin < wb || st.cur_bin >= we) {  // "Walker escaped its energy window"
        if (lane == 0) record_error(ctl, WLG_ERR_ESCAPED, w);
        failed = true;
    }
    const DeviceParams& P = v.p;
    double* fg = v.fields + static_cast<size_t>(st.slot) * ld;
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * ld;
    double f = lane < n ? fg[lane] : 0.0;                                  // field of site `lane`
    uint32_t down = __ballot_sync(kFull, lane < n && sg[lane] < 0);        // bit j: spin j is -1
    const Grid g = v.grid;
    const int gcount = static_cast<int>(g.count);
    const double neg_min_scaled = -g.minimum * g.inv_width;
    const uint64_t force_limit = P.force_after != 0 ? P.force_after : ~0ULL;

    uint32_t hq = 0, avail = 0;  // draw index of the current site; draws [0, avail) are in the ring
    auto ensure = [&](uint32_t need) -> bool {  // draws [0, need] available
        for (uint32_t polls = 0; polls < kWindowWaitPolls; ++polls) {
            avail = __shfl_sync(kFull, ld_acquire_u32(produced_addr), 0);
            if (static_cast<int32_t>(need - avail) < 0) return true;
        }
        return false;
    };
    // The producer needs to know only when a whole batch of 32 draws has been consumed (its
    // room test is per batch), so the consumed count is published when the draw index has
    // entered a new batch (hq and the last published count differ above bit 4), from the rare
    // branch at the top of an attempt, not after every attempt.
    uint32_t published = 0;
    int i = 0, c1 = 0, c2 = 0;  // current site; candidates for the next one
    double h = 0.0, lnu = 0.0;  // field of the current site; log uniform of draw hq+1
    if (!failed) {
        if (!ensure(4)) {
            if (lane == 0) record_error(ctl, WLG_ERR_TIMEOUT, w);
            failed = true;
        } else {
            i = rec_site[0];
            c1 = rec_site[1];
            c2 = rec_site[2];
            lnu = rec_lnu[1];
            h = __shfl_sync(kFull, f, i < 0 ? 0 : i);
        }
    }

    uint32_t ran = 0;
    for (uint32_t epoch = 0; epoch < epochs; ++epoch) {
        if (!failed) {
            uint32_t batch;
            {
                uint64_t b = P.exchange_interval;
                if (P.max_attempts) {
                    const uint64_t remaining = st.attempted < P.max_attempts ? P.max_attempts - st.attempted : 0;
                    b = remaining < b ? remaining : b;
                }
                batch = static_cast<uint32_t>(b < 0xffffffffULL ? b : 0xffffffffULL);
            }
            double E = st.energy;
            double factor = st.factor;
            int32_t stage = st.stage;
            const uint64_t att0 = st.attempted;
            uint64_t since = st.attempted - st.last_accepted;
            uint32_t n_acc = 0, n_forced = 0;
            uint64_t active_count = st.active_count;
            int cur = st.cur_bin;
            double lg_cur = lg_s[cur - wb];
            uint64_t active_before = 0;
            if (stage != kInverseTime) {
                for (int b = lane; b < nbins; b += 32) active_before += act_s[b] ? 1 : 0;
                active_before = warp_sum_u64(active_before);
            }

            // The attempts of one batch; kIT selects the 1/t stage (per-attempt factor and
            // active count) or the Wang-Landau / frozen stages (constant factor); kForce the
            // forced acceptance (force_accept_after_attempts != 0), without which only the last
            // acceptance is tracked.
            auto run = [&](auto it_tag, auto force_tag) {
                constexpr bool kIT = decltype(it_tag)::value;
                constexpr bool kForce = decltype(force_tag)::value;
                uint32_t acc_t = 0;  // without forced acceptance: the t of the last acceptance
                uint32_t active32 = static_cast<uint32_t>(active_count);  // at most the window's bins
                // the current bin's histogram delta and visited flag, kept in registers like its
                // log g (lg_cur); the shared copies are written every attempt and read only for
                // the proposed bin, together with its log g
                uint32_t hcnt = hd[cur - wb];
                bool cur_vis = act_s[cur - wb] != 0;
                const bool frozen = stage == kFrozen;
                InverseTimeTable32 itt;  // the 1/t factors of the coming attempts
                // 1/t stage: an attempt's factor and freeze are applied to log g of its bin at the point
                // where the next attempt first reads log g, so the factor's shuffle is not waited for
                double lg_base_p = 0.0, f_p = 0.0;
                bool pend = false;
                for (uint32_t t = 0; t < batch;) {
                    // the rare cases share one branch: a consumed count to publish, draws not yet
                    // in the ring, a site draw that bounded() rejected, and (1/t stage) a refresh
                    // of the factor table (every 32 attempts, or when the active count changed)
                    const bool publish = (hq ^ published) >= 32u;
                    const bool wait_draws = static_cast<int32_t>(hq + 4 - avail) >= 0;
                    bool rare = publish || wait_draws || i < 0;
                    if constexpr (kIT) rare = rare || itt.next >= 32 || active32 != itt.active;
                    if (rare) {
                        if (publish) {
                            __syncwarp();  // every lane's reads of the consumed records come first
                            if (lane == 0) st_release_u32(consumed_addr, hq);
                            published = hq;
                        }
                        if (wait_draws && !ensure(hq + 4)) {
                            failed = true;
                            break;
                        }
                        if (i < 0) {  // bounded() rejects draw hq; the next draw is the site
                            hq += 1;
                            i = c1;
                            h = __shfl_sync(kFull, f, i < 0 ? 0 : i);
                            c1 = c2;
                            c2 = rec_site[(hq + 2) & kWindowRingMask];
                            lnu = rec_lnu[(hq + 1) & kWindowRingMask];
                            continue;
                        }
                        if constexpr (kIT) {
                            if (itt.next >= 32 || active32 != itt.active)
                                inverse_time_refresh(itt, att0 + st.time_offset + t, active32, lane);
                        }
                    }
                    // loads: the couplings of the site, the candidates' fields, the next records
                    const int c1l = c1 < 0 ? 0 : c1, c2l = c2 < 0 ? 0 : c2;
                    const double* Ji = J_s + i * ld;
                    const double jr = lane < ld ? Ji[lane] : 0.0;
                    const double r1 = Ji[c1l], r2 = Ji[c2l];
                    const double fc1 = __shfl_sync(kFull, f, c1l), fc2 = __shfl_sync(kFull, f, c2l);
                    const int r3 = rec_site[(hq + 3) & kWindowRingMask], r4 = rec_site[(hq + 4) & kWindowRingMask];
                    const double l2 = rec_lnu[(hq + 2) & kWindowRingMask], l3 = rec_lnu[(hq + 3) & kWindowRingMask];

                    // the decision (attempt_flip, src/wang_landau.cpp:244-262)
                    const double m = ((down >> i) & 1u) ? 2.0 : -2.0;  // -2 * spin
                    const double Ep = fma(m, h, E);
                    const bool in_range = Ep >= g.minimum && Ep <= g.maximum;
                    const double qv = kPow2 ? fma(Ep, g.inv_width, neg_min_scaled) : (Ep - g.minimum) / g.width;
                    int nb = in_range ? bin_floor(qv) : -1;
                    nb = (nb == gcount && Ep == g.maximum) ? gcount - 1 : nb;
                    const bool in_window = nb >= wb && nb < we;
                    const int nl = in_window ? nb - wb : 0;
                    const double lg_load = lg_s[nl];
                    const uint32_t hd_load = hd[nl];
                    const bool act_load = act_s[nl] != 0;
                    if (kIT) {  // the previous attempt's factor (update_inverse_time_factor) and log g update
                        const bool frz = pend && f_p <= P.final_factor;
                        stage = frz ? kFrozen : stage;
                        factor = pend ? f_p : factor;
                        lg_cur = pend ? (frz ? lg_base_p : lg_base_p + f_p) : lg_cur;
                        pend = false;
                    }
                    const double lg_new = nb == cur ? lg_cur : lg_load;
                    const double log_ratio = lg_cur - lg_new;
                    const bool det = log_ratio >= 0.0;
                    const bool forced = kForce && !det && since >= force_limit;
                    const bool need_u = in_window && !det && !forced;
                    const bool accepted = in_window && (det || forced || lnu < log_ratio);

                    // add_flip_delta on every site; the next attempt's site and field
                    const double m_eff = accepted ? m : 0.0;
                    f = fma(m_eff, jr, f);
                    const int c = need_u ? c2 : c1;
                    const double h_next = fma(m_eff, need_u ? r2 : r1, need_u ? fc2 : fc1);
                    down ^= accepted ? (1u << i) : 0u;
                    E = accepted ? Ep : E;
                    n_acc += accepted ? 1u : 0u;
                    if constexpr (kForce) {
                        since = accepted ? 0 : since + 1;
                        n_forced += (accepted && forced) ? 1u : 0u;
                    }
                    ++t;
                    if constexpr (!kForce) acc_t = accepted ? t : acc_t;

                    // update_inverse_time_factor then update_current_bin (src/wang_landau.cpp:277-278)
                    if (kIT) {  // resolved at the next read of log g; nothing pends once frozen
                        f_p = inverse_time_factor_next(itt, active32, factor);
                        pend = stage == kInverseTime;
                    }
                    const bool move = accepted && nb != cur;
                    const int ncur = move ? nb : cur;
                    const double lg_base = move ? lg_new : lg_cur;
                    if (kIT) {
                        const bool visited = move ? act_load : cur_vis;
                        active32 += visited ? 0u : 1u;
                    }
                    hcnt = (move ? hd_load : hcnt) + 1u;
                    // every lane stores the same values (no branch, no atomic, no warp barrier:
                    // each lane reads back only what it has stored itself)
                    lg_s[cur - wb] = lg_cur;
                    hd[ncur - wb] = hcnt;
                    act_s[ncur - wb] = 1;
                    cur_vis = true;
                    cur = ncur;
                    if (kIT) {
                        lg_base_p = lg_base;
                        lg_cur = lg_base;  // plus the factor once it is resolved (pend)
                    } else {
                        lg_cur = frozen ? lg_base : lg_base + factor;
                    }
                    hq += need_u ? 2u : 1u;
                    i = c;
                    h = h_next;
                    c1 = need_u ? r3 : c2;
                    c2 = need_u ? r4 : r3;
                    lnu = need_u ? l3 : l2;
                }
                if constexpr (!kForce) since = n_acc ? static_cast<uint64_t>(batch - acc_t) : since + batch;
                if (kIT) active_count = active32;
                if (kIT && pend) {  // the last attempt's factor
                    const bool frz = f_p <= P.final_factor;
                    stage = frz ? kFrozen : stage;
                    factor = f_p;
                    lg_cur = frz ? lg_base_p : lg_base_p + f_p;
                }
            };
            if (P.force_after != 0) {
                if (stage == kInverseTime) run(std::true_type{}, std::true_type{});
                else run(std::false_type{}, std::true_type{});
            } else {
                if (stage == kInverseTime) run(std::true_type{}, std::false_type{});
                else run(std::false_type{}, std::false_type{});
            }

            if (failed) {
                if (lane == 0) record_error(ctl, WLG_ERR_TIMEOUT, w);
            } else {
                if (lane == 0) lg_s[cur - wb] = lg_cur;
                __syncwarp();
                // fold the histogram deltas into H; the Wang-Landau count of active bins from the mask
                uint64_t active_after = 0;
                for (int b = lane; b < nbins; b += 32) {
                    h_s[b] += hd[b];
                    hd[b] = 0;
                    active_after += act_s[b] ? 1 : 0;
                }
                active_after = warp_sum_u64(active_after);
                if (st.stage != kInverseTime) active_count += active_after - active_before;
                __syncwarp();
                st.energy = E;
                st.factor = factor;
                st.stage = stage;
                st.attempted = att0 + batch;
                st.accepted += n_acc;
                st.forced += n_forced;
                st.last_accepted = st.attempted - since;
                st.active_count = active_count;
                st.cur_bin = cur;
                if (st.stage == kWangLandau) {  // the check of run_rewl (src/parallel.cpp:395-407)
                    const bool at_limit = P.max_attempts != 0 && st.attempted >= P.max_attempts;
                    if (st.attempted - st.last_check >= P.check_interval || at_limit) {
                        st.last_check = st.attempted;
                        const HistStats hs = warp_histogram_statistics(h_s, act_s, nbins, st.active_count, lane);
                        st.last_flatness = P.inverse_time ? hs.coverage : hs.min_over_mean;
                        if (stats_ready(hs, st.stage, P)) warp_begin_next_iteration(st, h_s, nullptr, nbins, P, lane);
                    }
                }
                if (lane == 0) {
                    if (st.stage == kFrozen) atomicAdd(&sc[1], 1);
                    if (P.max_attempts != 0 && st.attempted >= P.max_attempts) atomicAdd(&sc[2], 1);
                }
            }
        }
        if (failed && lane == 0) atomicExch(&sc[3], 1);
        walkers_barrier(32 * W);
        if (warp == 0 && lane == 0) {  // the termination test of run_rewl (src/parallel.cpp:527-533)
            const bool all_frozen = sc[1] == W;
            const bool limit = P.max_attempts != 0 && sc[2] == W;
            sc[0] = (all_frozen || limit || sc[3] != 0) ? 1 : 0;
            sc[1] = 0;
            sc[2] = 0;
        }
        ++ran;
        walkers_barrier(32 * W);
        if (sc[0]) break;
    }

    __syncwarp();
    if (lane == 0) {
        st_release_u32(consumed_addr, hq);
        st_release_u32(stop_addr, 1u);
    }
    __syncthreads();  // the producers have stopped and left their generator state
    if (!failed && wctl[3] != 0) {
        if (lane == 0) record_error(ctl, WLG_ERR_TIMEOUT, w);
        failed = true;
    }
    if (threadIdx.x == 0) {
        ctl->epoch += ran;
        if (sc[0]) ctl->done = 1;
        ctl->frozen = 0;
        ctl->at_limit = 0;
    }
    if (failed) return;
    Rng rng{wrng[0], wrng[1], wrng[2], wrng[3]};
    for (uint32_t k = hq; k != wctl[1]; ++k) rng_step_back(rng);  // back over the unconsumed draws
    st.rng[0] = rng.s0;
    st.rng[1] = rng.s1;
    st.rng[2] = rng.s2;
    st.rng[3] = rng.s3;
    if (lane < n) {
        fg[lane] = f;
        sg[lane] = static_cast<int8_t>(((down >> lane) & 1u) ? -1 : 1);
    }
    for (int b = lane; b < nbins; b += 32) {
        v.log_g[boff + b] = lg_s[b];
        v.hist[boff + b] = h_s[b];
        v.active[boff + b] = act_s[b];
    }
    if (lane == 0) v.ws[w] = st;
}

using WindowFn = void (*)(EngineView, uint32_t);

template <bool kPow2>
WindowFn window_fn() {
    static bool configured = false;
    if (!configured) {
        check_cuda(cudaFuncSetAttribute(reinterpret_cast<const void*>(&sweep_window_kernel<kPow2>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    return &sweep_window_kernel<kPow2>;
}

}  // namespace

bool window_sweep_fits(const EngineView& v) {
    return !v.csr && v.precision == WLG_PRECISION_FP64 && !v.p.collect && !v.p.nalivaiko && v.windows == 1 &&
           v.walkers >= 1 && v.walkers <= kWindowMaxWalkers && v.n >= 1 && v.n <= 32 && v.ld <= 32 &&
           window_layout(v.ld, v.max_window_bins, v.walkers).total <= 200 * 1024;
}

void launch_sweep_window(const EngineView& v, uint32_t epochs, cudaStream_t stream) {
    const size_t bytes = window_layout(v.ld, v.max_window_bins, v.walkers).total;
    WindowFn fn = v.grid.pow2_width ? window_fn<true>() : window_fn<false>();
    fn<<<1, static_cast<unsigned>(64 * v.walkers), bytes, stream>>>(v, epochs);
    check_cuda(cudaGetLastError(), "sweep_window_kernel");
}

}  // namespace wlg
