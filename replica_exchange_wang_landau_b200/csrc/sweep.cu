// sweep.cu — the dense REWL sweep: WangLandauWalker::run_attempts / attempt_flip
// (src/wang_landau.cpp:244-315) for one batch of exchange_interval attempts, then the
// walker-local flatness / 1/t check of run_rewl (src/parallel.cpp:395-407).
//
// One warp owns one walker (one CTA per walker: with 128 walkers on 148 SMs every walker has
// an SM to itself).  The walker's local fields, spins and window slice of log_g / H / active
// live in shared memory, and the J rows it will need arrive in a shared-memory ring ahead of
// time:
//
// * The random site of an attempt is the next unconsumed draw of the walker's xoshiro
//   stream, whatever the walk did before, so the warp generates its draws kSlots ahead and,
//   for every draw, starts a bulk asynchronous copy (cp.async.bulk, completion counted on an
//   mbarrier) of the J row of the site that draw would select.  A draw consumed as a site
//   whose flip is accepted finds its row on chip; a draw consumed as the acceptance uniform
//   just frees its slot.  At the end of the batch the generator is stepped back over the
//   draws still queued (rng_step_back), so the stored RNG state is the reference's.
// * All 32 lanes evaluate the scalar decision chain redundantly (identical registers, no
//   shuffles); the lanes split the N-element field update.  One elected lane issues the
//   copies (elect.sync, no branch).
// * Every mbarrier wait is bounded; on timeout the walker records WLG_ERR_TIMEOUT, drains its
//   outstanding copies (bounded again) and returns without writing its state back.
//
// The arithmetic is the reference's, operation for operation (see walker.cu for the shared
// argument about fma(m, J, h) with m = +-2 and the power-of-two bin width).
#include <type_traits>

#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

namespace {

constexpr int kSlots = 4;
constexpr uint32_t kWaitPolls = 1u << 18;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Warp-uniform bounded wait for the completion of phase `parity` of one barrier.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (__all_sync(kFull, mbar_try(bar, parity))) return true;
    for (uint32_t k = 1; k < kWaitPolls; ++k)
        if (__all_sync(kFull, mbar_try(bar, parity))) return true;
    return false;
}
// One elected lane arms the slot's barrier with the row size and starts the row copy.
// `fence` orders this warp's earlier shared-memory reads of the slot before the copy.
__device__ __forceinline__ void issue_row(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar, bool fence) {
    if (fence) {
        asm volatile(
            "{\n .reg .pred p;\n elect.sync _|p, 0xffffffff;\n"
            " @p fence.proxy.async.shared::cta;\n"
            " @p mbarrier.arrive.expect_tx.shared::cta.b64 _, [%3], %2;\n"
            " @p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n}" ::"r"(dst),
            "l"(src), "r"(bytes), "r"(bar)
            : "memory");
    } else {
        asm volatile(
            "{\n .reg .pred p;\n elect.sync _|p, 0xffffffff;\n"
            " @p mbarrier.arrive.expect_tx.shared::cta.b64 _, [%3], %2;\n"
            " @p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n}" ::"r"(dst),
            "l"(src), "r"(bytes), "r"(bar)
            : "memory");
    }
}

struct RingLayout {
    size_t ring, bars, base, total;
};
__host__ __device__ inline RingLayout ring_layout(int ld, int mwb, bool features, size_t jbytes) {
    RingLayout L;
    size_t at = 0;
    L.ring = at;
    at += kSlots * round16(static_cast<size_t>(ld) * jbytes);
    L.bars = at;
    at += round16(kSlots * 8);
    L.base = at;
    at += smem_layout(ld, mwb, true, features).total;
    L.total = at;
    return L;
}

template <int kPrec> struct CouplingType;
template <> struct CouplingType<WLG_PRECISION_FP64> { using T = double; };
template <> struct CouplingType<WLG_PRECISION_FP32> { using T = float; };
template <> struct CouplingType<WLG_PRECISION_BF16> { using T = __nv_bfloat16; };

// fields[j] += m * row[j] (add_flip_delta, src/physics.cpp:190-195) from a row in shared
// memory; m * row[j] is exact (m = +-2, times the BF16 row scale), so fma rounds once as
// the reference's multiply-then-add does.  The fields are updated in groups of eight double2
// per lane (lane-contiguous, so every access is conflict-free), all of a group's loads issued
// before its stores, since a shared-memory load issued behind pending stores of the same warp
// waits for them (FP64, N = 2458: 138 -> 189 M attempts/s).  FP32 and BF16 rows are read as
// the pair of couplings of each double2 of fields (float2 / one 32-bit word) and widened
// exactly to double.
template <int kPrec>
__device__ __forceinline__ void row_update(const void* row_smem, int ld, double m, double* f, int lane) {
    double2* f2 = reinterpret_cast<double2*>(f);
    constexpr int kGroup = 8;  // double2 per lane per group (16 measured slower for FP64)
    const int n2 = ld >> 1;
    for (int base = 0; base < n2; base += 32 * kGroup) {
        double2 a[kGroup], h[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; ++q) {
            const int k = base + lane + 32 * q;
            if (k < n2) {
                if constexpr (kPrec == WLG_PRECISION_FP64) {
                    a[q] = reinterpret_cast<const double2*>(row_smem)[k];
                } else if constexpr (kPrec == WLG_PRECISION_FP32) {
                    const float2 p = reinterpret_cast<const float2*>(row_smem)[k];
                    a[q] = make_double2(static_cast<double>(p.x), static_cast<double>(p.y));
                } else {  // BF16 pair: element 2k in the low half of the word, 2k+1 in the high half
                    const uint32_t w = reinterpret_cast<const uint32_t*>(row_smem)[k];
                    a[q] = make_double2(static_cast<double>(__uint_as_float(w << 16)),
                                        static_cast<double>(__uint_as_float(w & 0xffff0000u)));
                }
                h[q] = f2[k];
            }
        }
#pragma unroll
        for (int q = 0; q < kGroup; ++q) {
            const int k = base + lane + 32 * q;
            if (k < n2) {
                h[q].x = fma(m, a[q].x, h[q].x);
                h[q].y = fma(m, a[q].y, h[q].y);
                f2[k] = h[q];
            }
        }
    }
}

template <int kPrec, bool kFeat>
__global__ void __launch_bounds__(32, 1) sweep_dense_kernel(EngineView v, WalkArgs a) {
    using JT = typename CouplingType<kPrec>::T;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    if (static_cast<int>(blockIdx.x) >= a.count) return;
    const int w = a.first + static_cast<int>(blockIdx.x);
    Control* ctl = v.ctl;
    if (a.epoch_mode && *reinterpret_cast<volatile int32_t*>(&ctl->done)) return;

    const RingLayout RL = ring_layout(v.ld, v.max_window_bins, kFeat, sizeof(JT));
    const SmemLayout L = smem_layout(v.ld, v.max_window_bins, true, kFeat);
    unsigned char* base = smem + RL.base;
    const JT* ring_rows = reinterpret_cast<const JT*>(smem + RL.ring);
    double* f = reinterpret_cast<double*>(base + L.fields);
    double* lg_s = reinterpret_cast<double*>(base + L.log_g);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(base + L.hist);
    double* sq_s = reinterpret_cast<double*>(base + L.sq);
    uint64_t* ds_s = reinterpret_cast<uint64_t*>(base + L.ds);
    int8_t* sp_s = reinterpret_cast<int8_t*>(base + L.spins);
    uint8_t* act_s = base + L.active;
    uint8_t* ref_s = base + L.refine;

    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    const size_t boff = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + static_cast<size_t>(wb);
    double* fg = v.fields + static_cast<size_t>(st.slot) * v.ld;
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * v.ld;
    const DeviceParams& P = v.p;
    const bool collect = kFeat && P.collect;
    const bool nalivaiko = kFeat && P.nalivaiko;

    if (st.cur_bin < wb || st.cur_bin >= we) {  // "Walker escaped its energy window"
        if (lane == 0) record_error(ctl, WLG_ERR_ESCAPED, w);
        return;
    }
    uint32_t batch;
    {
        uint64_t b = a.fixed_batch ? a.fixed_batch : P.exchange_interval;
        if (!a.fixed_batch && P.max_attempts) {
            const uint64_t remaining = st.attempted < P.max_attempts ? P.max_attempts - st.attempted : 0;
            b = remaining < b ? remaining : b;
        }
        batch = static_cast<uint32_t>(b < 0xffffffffULL ? b : 0xffffffffULL);
    }

    // ---- the row ring: barriers, then the first kSlots draws and their rows -------------
    const JT* J = kPrec == WLG_PRECISION_FP64   ? reinterpret_cast<const JT*>(v.J64)
                  : kPrec == WLG_PRECISION_FP32 ? reinterpret_cast<const JT*>(v.J32)
                                                : reinterpret_cast<const JT*>(v.J16);
    const uint32_t row_bytes = static_cast<uint32_t>(v.ld * sizeof(JT));
    const uint32_t ring_addr = smem_addr(smem + RL.ring);
    const uint32_t bar_addr = smem_addr(smem + RL.bars);
    if (lane == 0) {
        for (int s = 0; s < kSlots; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_addr + 8 * s) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};  // runs kSlots draws ahead of the walk
    uint64_t q0 = rng.next(), q1 = rng.next(), q2 = rng.next(), q3 = rng.next();
    issue_row(ring_addr + 0 * row_bytes, J + fast_mod(v.site_mod, q0) * v.ld, row_bytes, bar_addr + 0, false);
    issue_row(ring_addr + 1 * row_bytes, J + fast_mod(v.site_mod, q1) * v.ld, row_bytes, bar_addr + 8, false);
    issue_row(ring_addr + 2 * row_bytes, J + fast_mod(v.site_mod, q2) * v.ld, row_bytes, bar_addr + 16, false);
    issue_row(ring_addr + 3 * row_bytes, J + fast_mod(v.site_mod, q3) * v.ld, row_bytes, bar_addr + 24, false);
    uint32_t parity = 0;     // bit s: the phase parity the next wait on slot s expects
    uint32_t inflight = 0xF; // bit s: a copy into slot s has not been observed complete
    uint32_t head = 0;       // slot holding the row of q0
    bool failed = false;

    auto wait_slot = [&](uint32_t s) -> bool {
        if (!((inflight >> s) & 1u)) return true;
        if (!mbar_wait(bar_addr + 8 * s, (parity >> s) & 1u)) return false;
        inflight &= ~(1u << s);
        parity ^= 1u << s;
        return true;
    };
    // consume q0: its slot receives the row for the draw kSlots ahead
    auto advance = [&](bool fence) {
        if (!wait_slot(head)) {
            failed = true;
            return;
        }
        q0 = q1;
        q1 = q2;
        q2 = q3;
        q3 = rng.next();
        issue_row(ring_addr + head * row_bytes, J + fast_mod(v.site_mod, q3) * v.ld, row_bytes, bar_addr + 8 * head,
                  fence);
        inflight |= 1u << head;
        head = (head + 1) & (kSlots - 1);
    };

    // ---- stage the walker into shared memory (overlaps the first copies) --------------
    {
        const double2* src = reinterpret_cast<const double2*>(fg);
        double2* dst = reinterpret_cast<double2*>(f);
        for (int k = lane; k < (v.ld >> 1); k += 32) dst[k] = src[k];
        const int4* ssrc = reinterpret_cast<const int4*>(sg);
        int4* sdst = reinterpret_cast<int4*>(sp_s);
        for (int k = lane; k < (v.ld >> 4); k += 32) sdst[k] = ssrc[k];
    }
    for (int b = lane; b < nbins; b += 32) {
        lg_s[b] = v.log_g[boff + b];
        h_s[b] = v.hist[boff + b];
        act_s[b] = v.active[boff + b];
        if constexpr (kFeat) {
            ref_s[b] = v.refine[boff + b];
            if (collect) {
                sq_s[b] = v.sqdisp[boff + b];
                ds_s[b] = v.dsamples[boff + b];
            }
        }
    }
    __syncwarp();
    if (collect && st.rep_pending) {
        warp_update_representatives(v, w, st.energy, sp_s, lane);
        st.rep_pending = 0;
    }

    // ---- the walk -----------------------------------------------------------------------
    double E = st.energy;
    double factor = st.factor;
    int32_t stage = st.stage;
    const uint64_t att0 = st.attempted;
    uint64_t since = st.attempted - st.last_accepted;  // attempted - last_accepted_attempt
    uint32_t n_acc = 0, n_forced = 0;
    uint64_t active_count = st.active_count, refine_count = st.refine_count;
    int32_t rt_state = st.rt_state;
    uint64_t trips = st.round_trips;
    const double lower = window_lower(v, wb);
    const double upper = window_lower(v, we);
    const Grid g = v.grid;
    const int gcount = static_cast<int>(g.count);
    int cur = st.cur_bin;
    double lg_cur = lg_s[cur - wb];
    uint64_t hc_cur = h_s[cur - wb];
    bool act_cur = act_s[cur - wb] != 0;
    bool ref_cur = nalivaiko ? ref_s[cur - wb] != 0 : true;
    const uint64_t threshold = v.site_mod.threshold;
    InverseTimeTable itt;  // the 1/t factors of the coming attempts

    for (uint32_t t = 0; t < batch && !failed;) {
        if (q0 < threshold) {  // bounded() rejects this draw; the next one is the site
            advance(false);
            continue;
        }
        const int i = static_cast<int>(fast_mod(v.site_mod, q0));
        // BF16: the site's row scale, loaded before the decision so that an accepted flip does not wait for it
        const float row_scale = kPrec == WLG_PRECISION_BF16 ? __ldg(v.Jscale + i) : 1.0f;
        const uint32_t slot = head;
        const int8_t si = sp_s[i];
        const double m = -2.0 * static_cast<double>(si);
        const double delta = m * f[i];  // flip_delta: -2 s_i h_i, exact
        const double Ep = E + delta;
        // EnergyGrid::index restricted to the window: -1 when outside the grid
        int nb = -1;
        if (Ep >= g.minimum && Ep <= g.maximum) {
            const double off = Ep - g.minimum;
            nb = static_cast<int>(floor(g.pow2_width ? off * g.inv_width : off / g.width));
            if (nb == gcount && Ep == g.maximum) nb = gcount - 1;
        }
        const bool in_window = nb >= wb && nb < we;
        const int li = in_window ? nb - wb : 0;
        const double lg_new = nb == cur ? lg_cur : lg_s[li];
        const double log_ratio = lg_cur - lg_new;
        bool accepted = false, forced = false, used_uniform = false;
        if (in_window) {
            if (log_ratio >= 0.0) {
                accepted = true;
            } else if (P.force_after != 0 && since >= P.force_after) {
                accepted = forced = true;
            } else {
                used_uniform = true;
                accepted = log_uniform_below(to_uniform(q1), log_ratio);
            }
        }
        if (accepted) {
            double mm = m;
            if constexpr (kPrec == WLG_PRECISION_BF16) mm *= row_scale;
            if (!wait_slot(slot)) {
                failed = true;
                break;
            }
            row_update<kPrec>(ring_rows + static_cast<size_t>(slot) * v.ld, v.ld, mm, f, lane);
            if (lane == 0) sp_s[i] = static_cast<int8_t>(-si);
            E = Ep;
            ++n_acc;
            n_forced += forced ? 1u : 0u;
            since = 0;
            __syncwarp();  // every lane's reads of the row precede the fenced refill
        } else {
            ++since;
        }
        advance(accepted);                 // the site draw
        if (used_uniform) advance(false);  // the acceptance uniform
        if (collect && lane == 0) {
            const double displacement = accepted ? delta : 0.0;
            sq_s[cur - wb] += displacement * displacement;
            ++ds_s[cur - wb];
        }
        ++t;
        if (stage == kInverseTime) {  // update_inverse_time_factor
            factor = inverse_time_factor(itt, att0 + st.time_offset + t - 1, active_count, factor, lane);
            if (factor <= P.final_factor) stage = kFrozen;
        }
        if (accepted && nb != cur) {  // update_current_bin moves to the new bin
            if (lane == 0) {
                lg_s[cur - wb] = lg_cur;
                h_s[cur - wb] = hc_cur;
                act_s[cur - wb] = act_cur ? 1 : 0;
                if (nalivaiko) ref_s[cur - wb] = ref_cur ? 1 : 0;
            }
            cur = nb;
            lg_cur = lg_new;
            hc_cur = h_s[li];
            act_cur = act_s[li] != 0;
            ref_cur = nalivaiko ? ref_s[li] != 0 : true;
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
    // drain: no copy may land after the CTA exits
    for (uint32_t s = 0; s < kSlots; ++s)
        if (!wait_slot(s)) failed = true;
    if (failed) {
        if (lane == 0) record_error(ctl, WLG_ERR_TIMEOUT, w);
        return;
    }
    if (lane == 0) {
        lg_s[cur - wb] = lg_cur;
        h_s[cur - wb] = hc_cur;
        act_s[cur - wb] = act_cur ? 1 : 0;
        if (nalivaiko) ref_s[cur - wb] = ref_cur ? 1 : 0;
    }
    __syncwarp();
    for (int k = 0; k < kSlots; ++k) rng_step_back(rng);  // back over the queued, unconsumed draws

    st.rng[0] = rng.s0;
    st.rng[1] = rng.s1;
    st.rng[2] = rng.s2;
    st.rng[3] = rng.s3;
    st.energy = E;
    st.factor = factor;
    st.stage = stage;
    st.attempted = att0 + batch;
    st.accepted += n_acc;
    st.forced += n_forced;
    st.last_accepted = st.attempted - since;
    st.active_count = active_count;
    st.refine_count = refine_count;
    st.cur_bin = cur;
    st.rt_state = rt_state;
    st.round_trips = trips;

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
    {
        const double2* src = reinterpret_cast<const double2*>(f);
        double2* dst = reinterpret_cast<double2*>(fg);
        for (int k = lane; k < (v.ld >> 1); k += 32) dst[k] = src[k];
        const int4* ssrc = reinterpret_cast<const int4*>(sp_s);
        int4* sdst = reinterpret_cast<int4*>(sg);
        for (int k = lane; k < (v.ld >> 4); k += 32) sdst[k] = ssrc[k];
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

// ---- the split sweep (FP64 couplings, no pilot statistics, no Nalivaiko mask) ------------
//
// The same attempts as sweep_dense_kernel, with the work that does not depend on the walk
// moved to a second warp of the CTA, which the SM runs on another scheduler:
//
// * Warp 1 (the producer) generates the walker's draws in batches of kDrawBatch.  Every lane
//   steps the generator through the batch and lane j keeps draw j; for it, lane j stores in
//   ring entry k % Q the site the draw would select (-1 when bounded() rejects it) and
//   log(max(u, 2^-53)) of the uniform it would give (src/wang_landau.cpp:261), and starts
//   the bulk copy of that site's J row into the entry's row slot.  The batch's copies
//   complete one mbarrier.  The producer stays at most Q draws ahead of the walker, which
//   publishes with a release store, after every attempt, the draws it no longer needs.
// * Warp 0 (the walker) runs the decision chain and the bookkeeping.  It waits on a batch's
//   barrier only when its lookahead (up to draw hq+4, hq being the current site's draw)
//   enters that batch.
// * The next attempt's site is q1 = draw hq+1 or, when this attempt consumes the acceptance
//   uniform, q2 = draw hq+2.  The walker loads for both candidates their field, spin and the
//   J entries it needs before deciding, and after deciding forms the next attempt's field
//   with one fma.  The update of all N fields (add_flip_delta) is applied one attempt late,
//   off the chain: during attempt t the lanes add m_{t-1} * row_{t-1} to the fields they keep
//   in registers and write them through to shared memory at the end of the attempt, so
//   shared memory holds the fields up to attempt t-2 while t runs; a candidate's field is
//   then fma(m_t, J_t, fma(m_{t-1}, J_{t-1}, f)), the reference's two updates in order.  An
//   update with m_eff = 0 (rejected flip) changes no field, because a field is never -0.0
//   (sums start at +0.0 and a sum that reaches zero is +0.0), so the fields stay
//   bit-identical to the reference's.
// * Within an attempt every shared-memory load is issued before every store: a load issued
//   behind pending stores of the same warp waits for them, which serialised the chain.
// * Histogram increments go to a 32-bit shared-memory delta per bin (a reduction without
//   return) that is folded into H at the end of the batch.  In the Wang-Landau stage the
//   count of active bins is not read during the batch, so it is updated once, from the active
//   mask, at the end; in the 1/t stage it is maintained per attempt.
// * In the 1/t stage the factor active / attempted comes from a table of 32 quotients (one
//   division per 32 attempts, InverseTimeTable), and an attempt's factor and freeze test are
//   applied to log g of its bin where the next attempt first reads log g, so neither the
//   division nor the shuffle that reads the quotient sits on the attempt's chain.
// * The bin index of an in-range energy is the low word of (q + 2^52) added with rounding
//   toward -infinity (bin_floor), one add instead of a double-to-integer conversion.
// * At the end of the batch the walker publishes a stop flag; the producer waits for every
//   copy it started, and the generator is stepped back over the draws the walker did not
//   consume, so the stored RNG state is the reference's.  All waits are bounded: on timeout
//   the walker records WLG_ERR_TIMEOUT, the copies are drained (bounded again) and the
//   walker's state is not written back.
// Bit-exactness of the rearranged arithmetic: E + (-2s)h is evaluated as fma(m, h, E), equal
// because m*h (m = +-2) is exact; with a power-of-two bin width, (E' - min) / width is
// evaluated as fma(E', 1/width, -min/width), equal because scaling by a power of two is exact
// and commutes with rounding; log(max(u, 2^-53)) < log_ratio is evaluated with the CUDA log,
// whose result can differ from the C library's only in the last bit.

constexpr uint32_t kProducerPolls = 1u << 24;
constexpr int kDrawBatch = 4;  // draws per producer batch (one barrier per batch)
// The ring holds 2^kRL draws with their J rows (the staging depth; the autotuner chooses 4
// or 5).  At least 16: the walker reads up to draw hq+4 while it still holds the row of draw
// hq-1 or hq-2, and the producer must be able to complete the batch holding draw hq+4.
constexpr int kMinRingLog = 4;
constexpr int kMaxRingLog = 5;

struct SplitLayout {
    size_t ring, bars, lnu, rs, site, hd, ctl, base, total;
};
__host__ __device__ inline SplitLayout split_layout(int ld, int mwb, size_t jbytes, int ring_log) {
    const size_t q = size_t{1} << ring_log;
    SplitLayout L;
    size_t at = 0;
    L.ring = at; at += q * round16(static_cast<size_t>(ld) * jbytes);
    L.bars = at; at += round16((q / kDrawBatch) * 8);
    L.lnu = at; at += round16(q * 8);
    L.rs = at; at += round16(q * 8);  // BF16: the row scale of each draw's site
    L.site = at; at += round16(q * 4);
    L.hd = at; at += round16(static_cast<size_t>(mwb) * 4);
    L.ctl = at; at += 64;  // consumed, stop, producer status, produced, rng[4]
    L.base = at; at += smem_layout(ld, mwb, true, false).total;
    L.total = at;
    return L;
}

__device__ __forceinline__ void st_release_shared(uint32_t addr, uint32_t value) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(addr), "r"(value) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_shared(uint32_t addr) {
    uint32_t value;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(value) : "r"(addr) : "memory");
    return value;
}
// Non-blocking test of the completion of phase `parity` of one barrier.
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait of one thread for the completion of phase `parity` of one barrier.
__device__ __forceinline__ bool mbar_wait_thread(uint32_t bar, uint32_t parity) {
    for (uint32_t k = 0; k < kWaitPolls; ++k)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// One coupling of a row in shared memory, and the pair (2c, 2c+1), as exact doubles.
template <int kPrec>
__device__ __forceinline__ double coupling(const typename CouplingType<kPrec>::T* row, int j) {
    if constexpr (kPrec == WLG_PRECISION_FP64) return row[j];
    else if constexpr (kPrec == WLG_PRECISION_FP32) return static_cast<double>(row[j]);
    else return static_cast<double>(__bfloat162float(row[j]));
}
template <int kPrec>
__device__ __forceinline__ double2 coupling_pair(const typename CouplingType<kPrec>::T* row, int c) {
    if constexpr (kPrec == WLG_PRECISION_FP64) {
        return reinterpret_cast<const double2*>(row)[c];
    } else if constexpr (kPrec == WLG_PRECISION_FP32) {
        const float2 f = reinterpret_cast<const float2*>(row)[c];
        return make_double2(f.x, f.y);
    } else {
        const __nv_bfloat162 b = reinterpret_cast<const __nv_bfloat162*>(row)[c];
        return make_double2(__bfloat162float(b.x), __bfloat162float(b.y));
    }
}

// kExact: ld == 64 * kChunks, every chunk of every lane is inside the row.  Otherwise the lower
// half of the chunks still is (kChunks is the power of two at or above ceil(ld / 64)), and only
// the upper half is masked.
template <int kChunks, bool kPow2, int kPrec, int kRL, bool kExact>
__global__ void __launch_bounds__(64, 1) sweep_dense_split_kernel(EngineView v, WalkArgs a) {
    using JT = typename CouplingType<kPrec>::T;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int qlog = kRL;
    constexpr uint32_t qm = (1u << qlog) - 1u;
    constexpr int blog = qlog - 2;  // log2 of the number of batch barriers (kDrawBatch == 4)
    constexpr uint32_t bm = (1u << blog) - 1u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (static_cast<int>(blockIdx.x) >= a.count) return;
    const int w = a.first + static_cast<int>(blockIdx.x);
    Control* ctl = v.ctl;
    if (a.epoch_mode && *reinterpret_cast<volatile int32_t*>(&ctl->done)) return;

    const int ld = v.ld;
    const SplitLayout SL = split_layout(ld, v.max_window_bins, sizeof(JT), kRL);
    const SmemLayout L = smem_layout(ld, v.max_window_bins, true, false);
    const size_t row_stride = round16(static_cast<size_t>(ld) * sizeof(JT)) / sizeof(JT);  // elements
    const JT* ring = reinterpret_cast<const JT*>(smem + SL.ring);
    double* rec_lnu = reinterpret_cast<double*>(smem + SL.lnu);
    double* rec_rs = reinterpret_cast<double*>(smem + SL.rs);
    int32_t* rec_site = reinterpret_cast<int32_t*>(smem + SL.site);
    uint32_t* hd = reinterpret_cast<uint32_t*>(smem + SL.hd);
    uint32_t* sctl = reinterpret_cast<uint32_t*>(smem + SL.ctl);  // [0] consumed [1] stop [2] status [3] produced
    uint64_t* srng = reinterpret_cast<uint64_t*>(smem + SL.ctl + 32);
    unsigned char* base = smem + SL.base;
    double* f_s = reinterpret_cast<double*>(base + L.fields);
    double* lg_s = reinterpret_cast<double*>(base + L.log_g);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(base + L.hist);
    int8_t* sp_s = reinterpret_cast<int8_t*>(base + L.spins);
    uint8_t* act_s = base + L.active;
    const uint32_t ring_addr = smem_addr(smem + SL.ring);
    const uint32_t bar_addr = smem_addr(smem + SL.bars);
    const uint32_t consumed_addr = smem_addr(sctl), stop_addr = consumed_addr + 4;
    const uint32_t row_bytes = static_cast<uint32_t>(row_stride * sizeof(JT));

    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    if (st.cur_bin < wb || st.cur_bin >= we) {  // "Walker escaped its energy window"
        if (threadIdx.x == 0) record_error(ctl, WLG_ERR_ESCAPED, w);
        return;
    }
    const DeviceParams& P = v.p;
    uint32_t batch;
    {
        uint64_t b = a.fixed_batch ? a.fixed_batch : P.exchange_interval;
        if (!a.fixed_batch && P.max_attempts) {
            const uint64_t remaining = st.attempted < P.max_attempts ? P.max_attempts - st.attempted : 0;
            b = remaining < b ? remaining : b;
        }
        batch = static_cast<uint32_t>(b < 0xffffffffULL ? b : 0xffffffffULL);
    }
    const size_t boff = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + static_cast<size_t>(wb);
    double2* fg2 = reinterpret_cast<double2*>(v.fields + static_cast<size_t>(st.slot) * ld);
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * ld;
    const int ld2 = ld >> 1;
    // chunk k of this lane (column pair lane + 32 k) lies inside the row
    auto inside = [&](int k, int c) { return kExact || k < kChunks / 2 || c < ld2; };
    double2 fr[kChunks];
    double2* f2s = reinterpret_cast<double2*>(f_s);

    if (warp == 1) {
        if (lane == 0) {
            for (uint32_t s = 0; s <= bm; ++s)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_addr + 8 * s) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            sctl[0] = 0;
            sctl[1] = 0;
            sctl[2] = 0;
        }
        for (int b = lane; b < nbins; b += 32) hd[b] = 0;
    } else {
        // stage the walker: fields in registers (lane's chunks) and written through to smem
#pragma unroll
        for (int k = 0; k < kChunks; ++k) {
            const int c = lane + 32 * k;
            fr[k] = inside(k, c) ? fg2[c] : make_double2(0.0, 0.0);
            if (inside(k, c)) f2s[c] = fr[k];
        }
        const int4* ssrc = reinterpret_cast<const int4*>(sg);
        int4* sdst = reinterpret_cast<int4*>(sp_s);
        for (int k = lane; k < (ld >> 4); k += 32) sdst[k] = ssrc[k];
        for (int b = lane; b < nbins; b += 32) {
            lg_s[b] = v.log_g[boff + b];
            h_s[b] = v.hist[boff + b];
            act_s[b] = v.active[boff + b];
        }
    }
    __syncthreads();

    if (warp == 1) {
        // ---- producer: batches of kDrawBatch draws, lane j < kDrawBatch handles draw j ----
        const FastMod fm = v.site_mod;
        const JT* J = kPrec == WLG_PRECISION_FP64   ? reinterpret_cast<const JT*>(v.J64)
                      : kPrec == WLG_PRECISION_FP32 ? reinterpret_cast<const JT*>(v.J32)
                                                    : reinterpret_cast<const JT*>(v.J16);
        Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};
        uint32_t produced = 0, status = 0;
        // withhold_draws: publish nothing, so that the walker's bounded wait runs out
        for (bool open = P.withhold_draws == 0; open;) {
            uint32_t consumed = __shfl_sync(kFull, lane == 0 ? ld_acquire_shared(consumed_addr) : 0u, 0);
            if (produced + kDrawBatch - consumed > qm + 1) {  // no room for a batch yet
                uint32_t go = 0;
                if (lane == 0) {
                    for (uint32_t polls = 0; polls < kProducerPolls; ++polls) {
                        if (ld_acquire_shared(stop_addr)) break;
                        consumed = ld_acquire_shared(consumed_addr);
                        if (produced + kDrawBatch - consumed <= qm + 1) {
                            go = 1;
                            break;
                        }
                    }
                    if (!go && !ld_acquire_shared(stop_addr)) status = WLG_ERR_TIMEOUT;
                }
                if (!__shfl_sync(kFull, go, 0)) break;
            }
            __syncwarp();  // lane 0's acquire orders the walker's reads before this batch's writes
            uint64_t mine = 0;
#pragma unroll
            for (int j = 0; j < kDrawBatch; ++j) {
                const uint64_t d = rng.next();
                mine = lane == j ? d : mine;
            }
            const uint32_t k = produced + static_cast<uint32_t>(lane);
            const uint32_t e = k & qm;
            int site = 0;
            if (lane < kDrawBatch) {
                site = mine < fm.threshold ? -1 : static_cast<int>(fast_mod(fm, mine));
                rec_lnu[e] = log(fmax(to_uniform(mine), 0x1.0p-53));
                rec_site[e] = site;
                if constexpr (kPrec == WLG_PRECISION_BF16) rec_rs[e] = static_cast<double>(v.Jscale[site < 0 ? 0 : site]);
            }
            const uint32_t n = produced >> 2;  // batch index
            const uint32_t bar = bar_addr + 8 * (n & bm);
            __syncwarp();  // the batch's records are written before its barrier is armed
            if (lane == 0)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                             "r"(row_bytes * kDrawBatch)
                             : "memory");
            __syncwarp();
            if (lane < kDrawBatch) {
                const JT* src = J + static_cast<size_t>(site < 0 ? 0 : site) * ld;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        ring_addr + e * row_bytes),
                    "l"(src), "r"(row_bytes), "r"(bar)
                    : "memory");
            }
            produced += kDrawBatch;
        }
        // every copy started must land before the block exits: the latest batch of each
        // barrier is the only one whose copies can still be in flight
        if (lane == 0) {
            const uint32_t batches = produced >> 2;
            const uint32_t first = batches > bm ? batches - bm - 1 : 0;
            for (uint32_t n = first; n != batches; ++n)
                if (!mbar_wait_thread(bar_addr + 8 * (n & bm), (n >> blog) & 1u)) status = WLG_ERR_TIMEOUT;
            sctl[2] = status;
            sctl[3] = produced;
            srng[0] = rng.s0;
            srng[1] = rng.s1;
            srng[2] = rng.s2;
            srng[3] = rng.s3;
        }
        __syncthreads();
        return;
    }

    // ---- walker ----
    double E = st.energy;
    double factor = st.factor;
    int32_t stage = st.stage;
    const uint64_t att0 = st.attempted;
    uint64_t since = st.attempted - st.last_accepted;
    const uint64_t force_limit = P.force_after != 0 ? P.force_after : ~0ULL;
    uint32_t n_acc = 0, n_forced = 0;
    uint64_t active_count = st.active_count;
    const Grid g = v.grid;
    const int gcount = static_cast<int>(g.count);
    const double neg_min_scaled = -g.minimum * g.inv_width;
    int cur = st.cur_bin;
    double lg_cur = lg_s[cur - wb];
    bool failed = false;

    uint32_t hq = 0;        // draw index of the current site
    uint32_t ready_to = 0;  // draws [0, ready_to) are known to be in shared memory
    // make draws [0, need] available (false on timeout)
    auto ensure = [&](uint32_t need) -> bool {
        while (static_cast<int32_t>(need - ready_to) >= 0) {
            const uint32_t n = ready_to >> 2;
            if (!__all_sync(kFull, mbar_wait_thread(bar_addr + 8 * (n & bm), (n >> blog) & 1u))) return false;
            ready_to += kDrawBatch;
        }
        return true;
    };
    if (!ensure(4)) failed = true;
    int i = -1, si = 0, c1 = -1, c2 = -1;  // current site; candidates for the next one
    double h = 0.0, lnu = 0.0;             // field of the current site; log uniform of draw hq+1
    if (!failed) {
        i = rec_site[0];
        c1 = rec_site[1];
        c2 = rec_site[2];
        lnu = rec_lnu[1];
        if (i >= 0) {
            si = sp_s[i];
            h = f_s[i];
        }
    }
    // The field update of an attempt is applied during the next one: m_prev and prev_slot
    // are its factor (times the row scale for BF16) and row.  Shared memory holds the
    // fields up to the attempt before.
    double m_prev = 0.0;
    uint32_t prev_slot = 0;
    uint64_t active_before = 0;
    if (stage != kInverseTime) {
        for (int b = lane; b < nbins; b += 32) active_before += act_s[b] ? 1 : 0;
        active_before = warp_sum_u64(active_before);
    }

    // The attempts of one batch; kIT selects the 1/t stage (per-attempt factor and active
    // count) or the Wang-Landau / frozen stages (constant factor); kForce the forced acceptance
    // (force_accept_after_attempts != 0), without which only the last acceptance is tracked.
    auto run = [&](auto it_tag, auto force_tag) {
        constexpr bool kIT = decltype(it_tag)::value;
        constexpr bool kForce = decltype(force_tag)::value;
        uint32_t active32 = static_cast<uint32_t>(active_count);  // at most the window's bins
        uint32_t acc_t = 0;  // without forced acceptance: the t of the last acceptance
        const bool frozen = stage == kFrozen;
        InverseTimeTable32 itt;  // the 1/t factors of the coming attempts
        // 1/t stage: an attempt's factor and freeze are applied to log g of its bin at the point
        // where the next attempt first reads log g, so the factor's shuffle is not waited for
        double lg_base_p = 0.0, f_p = 0.0;
        bool pend = false;
        for (uint32_t t = 0; t < batch;) {
            // the two rare cases share one branch: draws still in flight, and a site draw that
            // bounded() rejected
            const bool wait_draws = static_cast<int32_t>(hq + 4 - ready_to) >= 0;
            if (wait_draws || i < 0) {
                if (wait_draws && !ensure(hq + 4)) {
                    failed = true;
                    break;
                }
                if (i < 0) {  // bounded() rejects draw hq; the next draw is the candidate site
                    const JT* prow = ring + static_cast<size_t>(prev_slot) * row_stride;
                    hq += 1;
                    i = c1;
                    if (i >= 0) {
                        si = sp_s[i];
                        h = fma(m_prev, coupling<kPrec>(prow, i), f_s[i]);
                    }
                    c1 = c2;
                    c2 = rec_site[(hq + 2) & qm];
                    lnu = rec_lnu[(hq + 1) & qm];
                    continue;
                }
            }
            // Look ahead at the next batch without blocking; the result is used at the end
            // of the attempt, so the test's latency overlaps the chain.  Every batch before
            // ready_to has completed, so that batch's barrier is in its phase or past it.
            const uint32_t next_batch = ready_to >> 2;
            const bool next_ready = mbar_test(bar_addr + 8 * (next_batch & bm), (next_batch >> blog) & 1u);
            const JT* prow = ring + static_cast<size_t>(prev_slot) * row_stride;
            const uint32_t slot = hq & qm;
            const JT* row = ring + static_cast<size_t>(slot) * row_stride;
            // loads: the next attempt's records, the candidates' fields, spins and couplings,
            // the previous attempt's row
            const int r3 = rec_site[(hq + 3) & qm], r4 = rec_site[(hq + 4) & qm];
            const double l2 = rec_lnu[(hq + 2) & qm], l3 = rec_lnu[(hq + 3) & qm];
            const int c1l = c1 < 0 ? 0 : c1, c2l = c2 < 0 ? 0 : c2;
            const double f1 = f_s[c1l], f2 = f_s[c2l];
            const int s1 = sp_s[c1l], s2 = sp_s[c2l];
            const double r1 = coupling<kPrec>(row, c1l), r2 = coupling<kPrec>(row, c2l);
            const double p1 = coupling<kPrec>(prow, c1l), p2 = coupling<kPrec>(prow, c2l);
            const double rscale = kPrec == WLG_PRECISION_BF16 ? rec_rs[slot] : 1.0;
            const double fc1 = fma(m_prev, p1, f1), fc2 = fma(m_prev, p2, f2);

            // the decision (attempt_flip, src/wang_landau.cpp:244-262)
            const double m = si > 0 ? -2.0 : 2.0;  // -2 * spin
            const double Ep = fma(m, h, E);
            const bool in_range = Ep >= g.minimum && Ep <= g.maximum;
            const double qv = kPow2 ? fma(Ep, g.inv_width, neg_min_scaled) : (Ep - g.minimum) / g.width;
            int nb = in_range ? bin_floor(qv) : -1;
            nb = (nb == gcount && Ep == g.maximum) ? gcount - 1 : nb;
            const bool in_window = nb >= wb && nb < we;
            const double lg_load = lg_s[in_window ? nb - wb : 0];
            // The row of the previous attempt is read only now: its 16-byte loads, issued
            // earlier, would queue ahead of the log g load on the chain.
            asm volatile("" ::: "memory");
            double2 rb[kChunks];
#pragma unroll
            for (int k = 0; k < kChunks; ++k) {
                const int cc = lane + 32 * k;
                rb[k] = inside(k, cc) ? coupling_pair<kPrec>(prow, cc) : make_double2(0.0, 0.0);
            }
            // the previous attempt's add_flip_delta (m_prev = 0 leaves every field unchanged)
#pragma unroll
            for (int k = 0; k < kChunks; ++k) {
                fr[k].x = fma(m_prev, rb[k].x, fr[k].x);
                fr[k].y = fma(m_prev, rb[k].y, fr[k].y);
            }
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

            // the next attempt's site, field and spin
            const int c = need_u ? c2 : c1;
            // m_eff * scale is exact (m = +-2, the scale is an FP32 value)
            const double m_eff = accepted ? (kPrec == WLG_PRECISION_BF16 ? m * rscale : m) : 0.0;
            const double h_next = fma(m_eff, need_u ? r2 : r1, need_u ? fc2 : fc1);
            const int s_next = (accepted && c == i) ? -si : (need_u ? s2 : s1);
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
                f_p = inverse_time_factor_select(itt, att0 + st.time_offset + t - 1, active32, factor, lane);
                pend = stage == kInverseTime;
            }
            const bool move = accepted && nb != cur;
            const int ncur = move ? nb : cur;
            const double lg_base = move ? lg_new : lg_cur;
            if (kIT) {
                const bool visited = act_s[ncur - wb] != 0;
                active32 += visited ? 0u : 1u;
            }

            // stores: the fields up to the previous attempt, the flipped spin, log g of the
            // bin left behind, the visit
#pragma unroll
            for (int k = 0; k < kChunks; ++k) {
                const int cc = lane + 32 * k;
                if (inside(k, cc)) f2s[cc] = fr[k];
            }
            // Wang-Landau stage: every lane stores the same values (no branch), lane 0 counts
            // the visit; the 1/t stage keeps them in lane 0's branch (measured faster there)
            if constexpr (!kIT) {
                sp_s[i] = static_cast<int8_t>(accepted ? -si : si);
                lg_s[cur - wb] = lg_cur;
                act_s[ncur - wb] = 1;
                if (lane == 0) atomicAdd(&hd[ncur - wb], 1u);
            } else if (lane == 0) {
                if (accepted) sp_s[i] = static_cast<int8_t>(-si);
                lg_s[cur - wb] = lg_cur;
                atomicAdd(&hd[ncur - wb], 1u);
                act_s[ncur - wb] = 1;
            }
            cur = ncur;
            if (kIT) {
                lg_base_p = lg_base;
                lg_cur = lg_base;  // plus the factor once it is resolved (pend)
            } else {
                lg_cur = frozen ? lg_base : lg_base + factor;
            }

            __syncwarp();  // the stores are visible to every lane
            // draws before this site are done (in the Wang-Landau stage every lane stores the value)
            if (!kIT || lane == 0) st_release_shared(consumed_addr, hq);
            hq += need_u ? 2u : 1u;
            i = c;
            si = s_next;
            h = h_next;
            c1 = need_u ? r3 : c2;
            c2 = need_u ? r4 : r3;
            lnu = need_u ? l3 : l2;
            m_prev = m_eff;
            prev_slot = slot;
            ready_to += __all_sync(kFull, next_ready) ? static_cast<uint32_t>(kDrawBatch) : 0u;
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
    if (!failed) {
        if (P.force_after != 0) {
            if (stage == kInverseTime) run(std::true_type{}, std::true_type{});
            else run(std::false_type{}, std::true_type{});
        } else {
            if (stage == kInverseTime) run(std::true_type{}, std::false_type{});
            else run(std::false_type{}, std::false_type{});
        }
    }
    if (!failed) {  // the last attempt's field update
        const JT* prow = ring + static_cast<size_t>(prev_slot) * row_stride;
#pragma unroll
        for (int k = 0; k < kChunks; ++k) {
            const int cc = lane + 32 * k;
            if (inside(k, cc)) {
                const double2 r = coupling_pair<kPrec>(prow, cc);
                fr[k].x = fma(m_prev, r.x, fr[k].x);
                fr[k].y = fma(m_prev, r.y, fr[k].y);
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        lg_s[cur - wb] = lg_cur;
        st_release_shared(consumed_addr, hq);
        st_release_shared(stop_addr, 1u);
    }
    __syncthreads();  // the producer has drained its copies and left its state
    if (failed || sctl[2] != 0) {
        if (lane == 0) record_error(ctl, WLG_ERR_TIMEOUT, w);
        return;
    }
    Rng rng{srng[0], srng[1], srng[2], srng[3]};
    for (uint32_t k = hq; k != sctl[3]; ++k) rng_step_back(rng);  // back over the unconsumed draws
    // fold the histogram deltas into H; the Wang-Landau count of active bins from the mask
    uint64_t active_after = 0;
    for (int b = lane; b < nbins; b += 32) {
        h_s[b] += hd[b];
        active_after += act_s[b] ? 1 : 0;
    }
    active_after = warp_sum_u64(active_after);
    if (st.stage != kInverseTime) active_count += active_after - active_before;
    __syncwarp();

    st.rng[0] = rng.s0;
    st.rng[1] = rng.s1;
    st.rng[2] = rng.s2;
    st.rng[3] = rng.s3;
    st.energy = E;
    st.factor = factor;
    st.stage = stage;
    st.attempted = att0 + batch;
    st.accepted += n_acc;
    st.forced += n_forced;
    st.last_accepted = st.attempted - since;
    st.active_count = active_count;
    st.cur_bin = cur;

    if (a.epoch_mode && st.stage == kWangLandau) {
        const bool at_limit = P.max_attempts != 0 && st.attempted >= P.max_attempts;
        if (st.attempted - st.last_check >= P.check_interval || at_limit) {
            st.last_check = st.attempted;
            const HistStats hs = warp_histogram_statistics(h_s, act_s, nbins, st.active_count, lane);
            st.last_flatness = P.inverse_time ? hs.coverage : hs.min_over_mean;
            if (stats_ready(hs, st.stage, P)) warp_begin_next_iteration(st, h_s, nullptr, nbins, P, lane);
        }
    }
#pragma unroll
    for (int k = 0; k < kChunks; ++k) {
        const int c = lane + 32 * k;
        if (inside(k, c)) fg2[c] = fr[k];
    }
    {
        const int4* ssrc = reinterpret_cast<const int4*>(sp_s);
        int4* sdst = reinterpret_cast<int4*>(sg);
        for (int k = lane; k < (ld >> 4); k += 32) sdst[k] = ssrc[k];
    }
    for (int b = lane; b < nbins; b += 32) {
        v.log_g[boff + b] = lg_s[b];
        v.hist[boff + b] = h_s[b];
        v.active[boff + b] = act_s[b];
    }
    if (lane == 0) {
        v.ws[w] = st;
        if (a.epoch_mode) {
            if (st.stage == kFrozen) atomicAdd(&ctl->frozen, 1u);
            if (P.max_attempts != 0 && st.attempted >= P.max_attempts) atomicAdd(&ctl->at_limit, 1u);
        }
    }
}

using SweepFn = void (*)(EngineView, WalkArgs);

template <int P, bool F>
SweepFn sweep_fn() {
    static bool configured = false;
    if (!configured) {
        check_cuda(cudaFuncSetAttribute(reinterpret_cast<const void*>(&sweep_dense_kernel<P, F>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    return &sweep_dense_kernel<P, F>;
}

}  // namespace

template <int K, bool kPow2, int kPrec, int kRL, bool kExact>
SweepFn split_fn_exact() {
    static bool configured = false;
    if (!configured) {
        check_cuda(cudaFuncSetAttribute(
                       reinterpret_cast<const void*>(&sweep_dense_split_kernel<K, kPow2, kPrec, kRL, kExact>),
                       cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    return &sweep_dense_split_kernel<K, kPow2, kPrec, kRL, kExact>;
}
template <int K, bool kPow2, int kPrec, int kRL>
SweepFn split_fn(int ld) {
    return ld == 64 * K ? split_fn_exact<K, kPow2, kPrec, kRL, true>() : split_fn_exact<K, kPow2, kPrec, kRL, false>();
}

// Chunks of 64 couplings per lane pass, rounded up to a power of two (unused chunks are
// masked off), for ld <= 1024.
template <bool kPow2, int kPrec, int kRL>
SweepFn pick_split_chunks(int ld) {
    const int chunks = (ld + 63) / 64;
    if (chunks <= 1) return split_fn<1, kPow2, kPrec, kRL>(ld);
    if (chunks <= 2) return split_fn<2, kPow2, kPrec, kRL>(ld);
    if (chunks <= 4) return split_fn<4, kPow2, kPrec, kRL>(ld);
    if (chunks <= 8) return split_fn<8, kPow2, kPrec, kRL>(ld);
    if (chunks <= 16) return split_fn<16, kPow2, kPrec, kRL>(ld);
    return nullptr;
}

template <int kPrec, int kRL>
SweepFn pick_split_precision(int ld, bool pow2_width) {
    return pow2_width ? pick_split_chunks<true, kPrec, kRL>(ld) : pick_split_chunks<false, kPrec, kRL>(ld);
}

template <int kRL>
SweepFn pick_split_ring(int ld, bool pow2_width, int precision) {
    if (precision == WLG_PRECISION_FP32) return pick_split_precision<WLG_PRECISION_FP32, kRL>(ld, pow2_width);
    if (precision == WLG_PRECISION_BF16) return pick_split_precision<WLG_PRECISION_BF16, kRL>(ld, pow2_width);
    return pick_split_precision<WLG_PRECISION_FP64, kRL>(ld, pow2_width);
}

// The split sweep for dense couplings with ld <= 1024, with a staging ring of 2^ring_log draws.
SweepFn pick_split(int ld, bool pow2_width, int precision, int ring_log) {
    return ring_log == kMaxRingLog ? pick_split_ring<kMaxRingLog>(ld, pow2_width, precision)
                                   : pick_split_ring<kMinRingLog>(ld, pow2_width, precision);
}

// Staging depths (log2 of the ring) the split sweep can run for this engine: those whose
// ring and window slice fit in one CTA's shared memory; empty when the split sweep does not
// serve it.
std::vector<int> split_ring_logs(const EngineView& v) {
    std::vector<int> out;
    const bool features = v.p.collect || v.p.nalivaiko;
    if (v.csr || features || v.ld > 1024) return out;
    const size_t jbytes = v.precision == WLG_PRECISION_FP64 ? 8 : v.precision == WLG_PRECISION_FP32 ? 4 : 2;
    for (int rl = kMinRingLog; rl <= kMaxRingLog; ++rl)
        if (split_layout(v.ld, v.max_window_bins, jbytes, rl).total <= 227 * 1024) out.push_back(rl);
    return out;
}

bool launch_sweep_dense(const EngineView& v, const WalkArgs& a, cudaStream_t stream) {
    const bool features = v.p.collect || v.p.nalivaiko;
    const size_t jbytes = v.precision == WLG_PRECISION_FP64 ? 8 : v.precision == WLG_PRECISION_FP32 ? 4 : 2;
    if (!features && v.ld <= 1024) {  // the split sweep
        int rl = v.split_ring_log == kMaxRingLog ? kMaxRingLog : kMinRingLog;
        if (split_layout(v.ld, v.max_window_bins, jbytes, rl).total > 227 * 1024) rl = kMinRingLog;
        SweepFn fn = pick_split(v.ld, v.grid.pow2_width != 0, v.precision, rl);
        const size_t split_bytes = split_layout(v.ld, v.max_window_bins, jbytes, rl).total;
        if (fn && split_bytes <= 227 * 1024) {
            fn<<<static_cast<unsigned>(a.count), 64, split_bytes, stream>>>(v, a);
            check_cuda(cudaGetLastError(), "sweep_dense_split_kernel");
            return true;
        }
    }
    const size_t bytes = ring_layout(v.ld, v.max_window_bins, features, jbytes).total;
    if (bytes > 227 * 1024) return false;
    SweepFn fn;
    if (v.precision == WLG_PRECISION_FP32)
        fn = features ? sweep_fn<WLG_PRECISION_FP32, true>() : sweep_fn<WLG_PRECISION_FP32, false>();
    else if (v.precision == WLG_PRECISION_BF16)
        fn = features ? sweep_fn<WLG_PRECISION_BF16, true>() : sweep_fn<WLG_PRECISION_BF16, false>();
    else
        fn = features ? sweep_fn<WLG_PRECISION_FP64, true>() : sweep_fn<WLG_PRECISION_FP64, false>();
    fn<<<static_cast<unsigned>(a.count), 32, bytes, stream>>>(v, a);
    check_cuda(cudaGetLastError(), "sweep_dense_kernel");
    return true;
}

}  // namespace wlg
