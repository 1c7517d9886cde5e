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
// the reference's multiply-then-add does.
template <int kPrec>
__device__ __forceinline__ void row_update(const void* row_smem, int ld, double m, double* f, int lane) {
    double2* f2 = reinterpret_cast<double2*>(f);
    if constexpr (kPrec == WLG_PRECISION_FP64) {
        const double2* r = reinterpret_cast<const double2*>(row_smem);
#pragma unroll 4
        for (int k = lane; k < (ld >> 1); k += 32) {
            const double2 a = r[k];
            double2 h = f2[k];
            h.x = fma(m, a.x, h.x);
            h.y = fma(m, a.y, h.y);
            f2[k] = h;
        }
    } else if constexpr (kPrec == WLG_PRECISION_FP32) {
        const float4* r = reinterpret_cast<const float4*>(row_smem);
#pragma unroll 2
        for (int k = lane; k < (ld >> 2); k += 32) {
            const float4 a = r[k];
            double2 h0 = f2[2 * k], h1 = f2[2 * k + 1];
            h0.x = fma(m, static_cast<double>(a.x), h0.x);
            h0.y = fma(m, static_cast<double>(a.y), h0.y);
            h1.x = fma(m, static_cast<double>(a.z), h1.x);
            h1.y = fma(m, static_cast<double>(a.w), h1.y);
            f2[2 * k] = h0;
            f2[2 * k + 1] = h1;
        }
    } else {
        const uint4* r = reinterpret_cast<const uint4*>(row_smem);
        for (int k = lane; k < (ld >> 3); k += 32) {
            const uint4 raw = r[k];
            const uint32_t words[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                double2 h = f2[4 * k + q];
                h.x = fma(m, static_cast<double>(__uint_as_float(words[q] << 16)), h.x);
                h.y = fma(m, static_cast<double>(__uint_as_float(words[q] & 0xffff0000u)), h.y);
                f2[4 * k + q] = h;
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

    for (uint32_t t = 0; t < batch && !failed;) {
        if (q0 < threshold) {  // bounded() rejects this draw; the next one is the site
            advance(false);
            continue;
        }
        const int i = static_cast<int>(fast_mod(v.site_mod, q0));
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
            if constexpr (kPrec == WLG_PRECISION_BF16) mm *= static_cast<double>(__ldg(v.Jscale + i));
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
            if (active_count != 0)
                factor = static_cast<double>(active_count) / static_cast<double>(att0 + t);
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

// ---- the lookahead sweep (FP64 couplings, no pilot statistics, no Nalivaiko mask) --------
//
// The same attempt as above, reorganised so that the N-element field update is not on the
// path from one attempt to the next, and so that the loop body is one branch-free block the
// compiler can schedule freely:
//
// * The next attempt's site is the draw after the site draw (q1) or, when this attempt
//   consumes the acceptance uniform, the one after that (q2).  Before deciding, the warp
//   loads for both candidates their field, spin and the J entry of the current site's row;
//   after deciding it forms the next attempt's field with one fma.
// * The update of all N fields then runs off the chain with m_eff = accepted ? m : 0: adding
//   m*0 changes no field, because a field is never -0.0 (sums start at +0.0 and a sum that
//   reaches zero is +0.0), so the fields stay bit-identical to the reference's.  Each lane
//   keeps its share of the fields in registers and writes them through to shared memory,
//   where the random single-field reads find them.
// * Rows arrive by per-lane cp.async copies, one commit group per attempt: each lane copies
//   exactly the 16-byte chunks of the row it will update.  A draw appended to the queue
//   reaches its head no earlier than four attempts later (it enters at position >= 6 and
//   moves by at most 2 per attempt), so "all but the 3 newest groups complete" covers the
//   site's row and "all but the 2 newest" the next draw's slot before it is reused; both
//   waits are single instructions.  When the uniform is not consumed, the second copy of the
//   attempt is a zero-size copy into a spare slot, so every attempt commits exactly one group.
// * The draws live in a small shared-memory queue; the generator runs kQueue draws ahead and
//   is stepped back over them at the end of the batch.
// Rare events (a rejected bounded() draw, an acceptance test inside the log margin, a first
// visit of a bin) take branches.

constexpr int kQueue = 8;       // draws generated ahead; row slots in the ring
constexpr int kQueueMask = 15;  // shared-memory draw queue of 16 entries

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int kPending> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(kPending) : "memory");
}

template <int kChunks>
__global__ void __launch_bounds__(32, 1) sweep_dense_fast_kernel(EngineView v, WalkArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    if (static_cast<int>(blockIdx.x) >= a.count) return;
    const int w = a.first + static_cast<int>(blockIdx.x);
    Control* ctl = v.ctl;
    if (a.epoch_mode && *reinterpret_cast<volatile int32_t*>(&ctl->done)) return;

    // carve-up: [kQueue + 1 row slots][draw queue][fields, log_g, H, spins, active]
    const int ld = v.ld;
    const size_t row_stride = static_cast<size_t>(ld) * 8;
    double* ring = reinterpret_cast<double*>(smem);
    uint64_t* dq = reinterpret_cast<uint64_t*>(smem + (kQueue + 1) * row_stride);
    unsigned char* base = smem + (kQueue + 1) * row_stride + (kQueueMask + 1) * 8;
    const SmemLayout L = smem_layout(ld, v.max_window_bins, true, false);
    double* f_s = reinterpret_cast<double*>(base + L.fields);
    double* lg_s = reinterpret_cast<double*>(base + L.log_g);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(base + L.hist);
    int8_t* sp_s = reinterpret_cast<int8_t*>(base + L.spins);
    uint8_t* act_s = base + L.active;

    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    const size_t boff = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + static_cast<size_t>(wb);
    double2* fg2 = reinterpret_cast<double2*>(v.fields + static_cast<size_t>(st.slot) * ld);
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * ld;
    const DeviceParams& P = v.p;
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

    const FastMod fm = v.site_mod;
    const double2* J2 = reinterpret_cast<const double2*>(v.J64);
    const int ld2 = ld >> 1;  // 16-byte chunks per row
    const uint32_t ring_addr = smem_addr(smem);
    const uint32_t rs = static_cast<uint32_t>(row_stride);
    // lane's chunks of a row: c = lane + 32k for k < kChunks, present when c < ld2
    auto copy_row = [&](uint32_t slot_addr, int site, uint32_t bytes) {
        const double2* src = J2 + static_cast<size_t>(site) * ld2;
#pragma unroll
        for (int k = 0; k < kChunks; ++k) {
            const int c = lane + 32 * k;
            if (c < ld2) cp_async16(slot_addr + 16u * c, src + c, bytes);
        }
    };
    Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};
    if (lane == 0)
        for (int k = 0; k < kQueue; ++k) dq[k] = 0;
    uint64_t first[kQueue];
#pragma unroll
    for (int k = 0; k < kQueue; ++k) {
        first[k] = rng.next();
        copy_row(ring_addr + k * rs, static_cast<int>(fast_mod(fm, first[k])), 16);
        cp_async_commit();
    }
    if (lane == 0)
        for (int k = 0; k < kQueue; ++k) dq[k] = first[k];

    // stage the walker: fields in registers (lane's chunks) and written through to smem
    double2 fr[kChunks];
    double2* f2s = reinterpret_cast<double2*>(f_s);
#pragma unroll
    for (int k = 0; k < kChunks; ++k) {
        const int c = lane + 32 * k;
        fr[k] = c < ld2 ? fg2[c] : make_double2(0.0, 0.0);
        if (c < ld2) f2s[c] = fr[k];
    }
    {
        const int4* ssrc = reinterpret_cast<const int4*>(sg);
        int4* sdst = reinterpret_cast<int4*>(sp_s);
        for (int k = lane; k < (ld >> 4); k += 32) sdst[k] = ssrc[k];
    }
    for (int b = lane; b < nbins; b += 32) {
        lg_s[b] = v.log_g[boff + b];
        h_s[b] = v.hist[boff + b];
        act_s[b] = v.active[boff + b];
    }
    __syncwarp();

    double E = st.energy;
    double factor = st.factor;
    int32_t stage = st.stage;
    const uint64_t att0 = st.attempted;
    uint64_t since = st.attempted - st.last_accepted;
    uint32_t n_acc = 0, n_forced = 0;
    uint64_t active_count = st.active_count;
    const Grid g = v.grid;
    const int gcount = static_cast<int>(g.count);
    int cur = st.cur_bin;
    double lg_cur = lg_s[cur - wb];
    const uint64_t threshold = fm.threshold;
    double factor_next = factor;
    if (stage == kInverseTime && active_count != 0)
        factor_next = static_cast<double>(active_count) / static_cast<double>(att0 + 1);
    const uint32_t spare_addr = ring_addr + kQueue * rs;

    uint32_t hq = 0;  // absolute queue index of the current site draw; its row is in slot hq % kQueue
    int i = static_cast<int>(fast_mod(fm, dq[0]));
    int si = sp_s[i];
    double h = f_s[i];
    uint64_t q0 = dq[0];

    for (uint32_t t = 0; t < batch;) {
        if (q0 < threshold) {  // rare: bounded() rejects this draw; the next one is the site
            cp_async_wait<0>();
            __syncwarp();
            const uint64_t d = rng.next();
            if (lane == 0) dq[(hq + kQueue) & kQueueMask] = d;
            copy_row(ring_addr + (hq & (kQueue - 1)) * rs, static_cast<int>(fast_mod(fm, d)), 16);
            cp_async_commit();
            ++hq;
            __syncwarp();
            q0 = dq[hq & kQueueMask];
            i = static_cast<int>(fast_mod(fm, q0));
            si = sp_s[i];
            h = f_s[i];
            continue;
        }
        const uint32_t slot = hq & (kQueue - 1);
        const double* row = ring + static_cast<size_t>(slot) * ld;
        const uint64_t q1 = dq[(hq + 1) & kQueueMask];
        const uint64_t q2 = dq[(hq + 2) & kQueueMask];
        cp_async_wait<3>();  // the site's row (and the previous attempt's field writes) are in
        __syncwarp();
        // lookahead: the two candidates for the next site
        const int c1 = static_cast<int>(fast_mod(fm, q1)), c2 = static_cast<int>(fast_mod(fm, q2));
        const double f1 = f_s[c1], f2 = f_s[c2];
        const int s1 = sp_s[c1], s2 = sp_s[c2];
        const double r1 = row[c1], r2 = row[c2];
        const double up = fmax(to_uniform(q1), 0x1.0p-53);
        const double est = static_cast<double>(__log2f(static_cast<float>(up))) * 0.6931471805599453;

        // the decision (attempt_flip, src/wang_landau.cpp:244-262)
        const double m = si > 0 ? -2.0 : 2.0;  // -2 * spin
        const double delta = m * h;
        const double Ep = E + delta;
        const double off = Ep - g.minimum;
        const double qv = g.pow2_width ? off * g.inv_width : off / g.width;
        int nb = (Ep >= g.minimum && Ep <= g.maximum) ? __double2int_rd(qv) : -1;
        nb = (nb == gcount && Ep == g.maximum) ? gcount - 1 : nb;
        const bool in_window = nb >= wb && nb < we;
        const double lg_load = lg_s[in_window ? nb - wb : 0];
        const double lg_new = nb == cur ? lg_cur : lg_load;
        const double log_ratio = lg_cur - lg_new;
        const bool det = log_ratio >= 0.0;
        const bool forced = !det && P.force_after != 0 && since >= P.force_after;
        const bool need_u = in_window && !det && !forced;
        bool u_ok = est < log_ratio - 1e-3;
        if (need_u && !u_ok && !(est > log_ratio + 1e-3)) u_ok = log(up) < log_ratio;  // inside the margin
        const bool accepted = in_window && (det || forced || u_ok);

        // the next attempt's site, field and spin
        const int c = need_u ? c2 : c1;
        const double m_eff = accepted ? m : 0.0;
        const double h_next = fma(m_eff, need_u ? r2 : r1, need_u ? f2 : f1);
        const int s_next = (accepted && c == i) ? -si : (need_u ? s2 : s1);

        // add_flip_delta off the chain (m_eff = 0 leaves every field unchanged)
        const double2* row2 = reinterpret_cast<const double2*>(row);
#pragma unroll
        for (int k = 0; k < kChunks; ++k) {
            const int cc = lane + 32 * k;
            if (cc < ld2) {
                const double2 r = row2[cc];
                fr[k].x = fma(m_eff, r.x, fr[k].x);
                fr[k].y = fma(m_eff, r.y, fr[k].y);
                f2s[cc] = fr[k];
            }
        }
        if (lane == 0 && accepted) sp_s[i] = static_cast<int8_t>(-si);
        E = accepted ? Ep : E;
        since = accepted ? 0 : since + 1;
        n_acc += accepted ? 1u : 0u;
        n_forced += (accepted && forced) ? 1u : 0u;
        ++t;

        // update_inverse_time_factor then update_current_bin (src/wang_landau.cpp:277-278)
        if (stage == kInverseTime) {
            factor = factor_next;
            if (factor <= P.final_factor) stage = kFrozen;
        }
        const bool move = accepted && nb != cur;
        if (lane == 0) lg_s[cur - wb] = lg_cur;
        const int ncur = move ? nb : cur;
        const double lg_base = move ? lg_new : lg_cur;
        const uint64_t hv = h_s[ncur - wb];
        const bool visited = act_s[ncur - wb] != 0;
        if (lane == 0) h_s[ncur - wb] = hv + 1;
        if (!visited) {  // rare: first visit of a bin
            if (lane == 0) act_s[ncur - wb] = 1;
            ++active_count;
        }
        cur = ncur;
        lg_cur = stage != kFrozen ? lg_base + factor : lg_base;
        if (stage == kInverseTime && active_count != 0)
            factor_next = static_cast<double>(active_count) / static_cast<double>(att0 + t + 1);

        // the consumed draws leave the queue; their slots get the draws kQueue ahead
        const uint64_t d1 = rng.next();
        Rng r2n = rng;
        const uint64_t d2 = r2n.next();
        rng.s0 = need_u ? r2n.s0 : rng.s0;
        rng.s1 = need_u ? r2n.s1 : rng.s1;
        rng.s2 = need_u ? r2n.s2 : rng.s2;
        rng.s3 = need_u ? r2n.s3 : rng.s3;
        if (lane == 0) {
            dq[(hq + kQueue) & kQueueMask] = d1;
            dq[(hq + kQueue + 1) & kQueueMask] = d2;
        }
        cp_async_wait<2>();  // the next draw's slot is free to reuse when the uniform was consumed
        __syncwarp();        // every lane has read the site's row and written its fields
        copy_row(ring_addr + slot * rs, static_cast<int>(fast_mod(fm, d1)), 16);
        copy_row(need_u ? ring_addr + ((hq + 1) & (kQueue - 1)) * rs : spare_addr, static_cast<int>(fast_mod(fm, d2)),
                 need_u ? 16u : 0u);
        cp_async_commit();
        hq += need_u ? 2u : 1u;
        q0 = need_u ? q2 : q1;
        i = c;
        si = s_next;
        h = h_next;
    }
    cp_async_wait<0>();  // no copy may land after the CTA exits
    if (lane == 0) lg_s[cur - wb] = lg_cur;
    __syncwarp();
    for (int k = 0; k < kQueue; ++k) rng_step_back(rng);  // back over the queued draws

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
        if (c < ld2) fg2[c] = fr[k];
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

size_t fast_smem_bytes(const EngineView& v) {
    return (kQueue + 1) * static_cast<size_t>(v.ld) * 8 + (kQueueMask + 1) * 8 +
           smem_layout(v.ld, v.max_window_bins, true, false).total;
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

template <int K>
SweepFn fast_fn() {
    static bool configured = false;
    if (!configured) {
        check_cuda(cudaFuncSetAttribute(reinterpret_cast<const void*>(&sweep_dense_fast_kernel<K>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    return &sweep_dense_fast_kernel<K>;
}

// The lookahead sweep for FP64 couplings with ld <= 1024 (chunks of 64 doubles per lane pass).
SweepFn pick_fast(int ld) {
    switch ((ld + 63) / 64) {
        case 1: return fast_fn<1>();
        case 2: return fast_fn<2>();
        case 3: return fast_fn<3>();
        case 4: return fast_fn<4>();
        case 5: return fast_fn<5>();
        case 6: return fast_fn<6>();
        case 7: return fast_fn<7>();
        case 8: return fast_fn<8>();
        case 9: return fast_fn<9>();
        case 10: return fast_fn<10>();
        case 11: return fast_fn<11>();
        case 12: return fast_fn<12>();
        case 13: return fast_fn<13>();
        case 14: return fast_fn<14>();
        case 15: return fast_fn<15>();
        case 16: return fast_fn<16>();
        default: return nullptr;
    }
}

bool launch_sweep_dense(const EngineView& v, const WalkArgs& a, cudaStream_t stream) {
    const bool features = v.p.collect || v.p.nalivaiko;
    const size_t jbytes = v.precision == WLG_PRECISION_FP64 ? 8 : v.precision == WLG_PRECISION_FP32 ? 4 : 2;
    if (!features && v.precision == WLG_PRECISION_FP64 && v.ld <= 1024) {  // the lookahead sweep
        const size_t fast_bytes = fast_smem_bytes(v);
        SweepFn fn = pick_fast(v.ld);
        if (fn && fast_bytes <= 227 * 1024) {
            fn<<<static_cast<unsigned>(a.count), 32, fast_bytes, stream>>>(v, a);
            check_cuda(cudaGetLastError(), "sweep_dense_fast_kernel");
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
