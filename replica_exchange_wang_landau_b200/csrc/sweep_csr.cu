// sweep_csr.cu — the REWL sweep for cutoff (CSR) couplings: WangLandauWalker::run_attempts /
// attempt_flip (src/wang_landau.cpp:244-315) with CsrCouplings::add_flip_delta
// (src/physics.cpp:231-236) for one batch of exchange_interval attempts, then the
// walker-local flatness / 1/t check of run_rewl (src/parallel.cpp:395-407).
//
// Large cutoff systems (a 32^3 lattice: 256 KB of FP64 fields and 32 KB of spins per walker,
// a thousand walkers) keep each walker's fields and spins in HBM; only the window slice of
// log g / H / visited lives in shared memory (a few KB), so every walker of a run is resident
// at once.  An attempt is then bound by memory latency, and the kernel is arranged so that an
// attempt waits for about one round trip:
//
// * The couplings are laid out as ELLPACK rows of 32*K entries (K = 1, 2, 4, 8; column -1 and
//   value 0 pad a row) with lane j holding entries j, j+32, ...: one coalesced load per
//   chunk and no row-pointer indirection.
// * The site of the next attempt is draw hq+1 or, when this attempt consumes the acceptance
//   uniform, draw hq+2 (the lookahead of the dense split sweep).  The site and both
//   candidates occupy three slots of a four-slot shared-memory ring: each slot receives by
//   cp.async (no register is the destination of a load in flight, so advancing the ring is
//   an index change) the site's couplings row, field and spin word, loaded at least one
//   attempt ahead and after the stores of every earlier flip.  A candidate is corrected for
//   the flip of the current attempt when it is a neighbour of the flipped site (a ballot over
//   the flipped row finds J_ic) and when it is the flipped site, so it equals the reference's
//   field and spin when it becomes the site: fma(m, J, f) with m = +-2 rounds the reference's
//   f + m*J once.
// * At the end of an attempt, after its stores, the warp copies the next site's neighbour
//   fields into its slot (speculatively: a rejected flip discards them); the next attempt
//   decides and on acceptance stores
//   fields[c] = fma(m, J_ic, fields[c]) for every neighbour c.  Each field changes at most
//   once per flip, so the order of the neighbour updates is immaterial.
// * The draws are generated 32 at a time, lane j keeping draw j with its site and the log
//   of its uniform, so the acceptance log is off the attempt's chain.
// * With pilot statistics on (an adaptive-window pilot), lane 0 adds each attempt's squared
//   displacement and sample to the old bin, and an accepted flip updates the round-trip state
//   and the representative configurations, in the reference's order.
// * All 32 lanes evaluate the decision chain redundantly; histogram increments go to a
//   32-bit shared-memory delta per bin that is folded into H at the end of the batch, and the
//   Wang-Landau count of active bins is updated once from the visited mask, as in the dense
//   split sweep.
// The kernel has no waits on other warps or kernels.  Bit-exactness of the rearranged
// arithmetic is argued where the dense sweeps use the same forms (E + (-2s)h as fma(m, h, E);
// the power-of-two bin index as fma(E', 1/width, -min/width); the acceptance test
// log(max(u, 2^-53)) < log_ratio with the CUDA log).
#include <type_traits>

#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

namespace {

// One ring slot: the couplings row (columns, values), the neighbour fields, the site's field
// and the 32-bit word of the spins array that holds its spin.
struct CsrSlot {
    size_t col, val, nf, f, sword, bytes;
};
__host__ __device__ inline CsrSlot csr_slot(int width, int vbytes) {
    CsrSlot S;
    size_t at = 0;
    S.col = at; at += static_cast<size_t>(width) * 4;
    S.val = at; at += static_cast<size_t>(width) * vbytes;
    S.nf = at; at += static_cast<size_t>(width) * 8;
    S.f = at; at += 8;
    S.sword = at; at += 8;
    S.bytes = round16(at);
    return S;
}
constexpr int kCsrSlots = 4;

struct CsrSweepLayout {
    size_t slots, log_g, hist, sq, ds, hd, active, total;
};
// `collect`: the pilot statistics of the window (squared displacements, sample counts)
__host__ __device__ inline CsrSweepLayout csr_sweep_layout(int mwb, int width, int vbytes, bool collect) {
    CsrSweepLayout L;
    size_t at = 0;
    L.slots = at; at += kCsrSlots * csr_slot(width, vbytes).bytes;
    L.log_g = at; at += round16(static_cast<size_t>(mwb) * 8);
    L.hist = at; at += round16(static_cast<size_t>(mwb) * 8);
    L.sq = at; at += collect ? round16(static_cast<size_t>(mwb) * 8) : 0;
    L.ds = at; at += collect ? round16(static_cast<size_t>(mwb) * 8) : 0;
    L.hd = at; at += round16(static_cast<size_t>(mwb) * 4);
    L.active = at; at += round16(static_cast<size_t>(mwb));
    L.total = at;
    return L;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// This thread's copies, all but the newest N groups, have landed.
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int kPrec> struct EllValue { using T = double; };
template <> struct EllValue<WLG_PRECISION_FP32> { using T = float; };

template <int kPrec>
__device__ __forceinline__ const typename EllValue<kPrec>::T* ell_values(const EngineView& v) {
    if constexpr (kPrec == WLG_PRECISION_FP32) return v.ell_val32;
    else return v.ell_val64;
}

template <int kK, bool kPow2, int kPrec, bool kCollect>
__global__ void __launch_bounds__(256, 1) sweep_csr_kernel(EngineView v, WalkArgs a) {
    using VT = typename EllValue<kPrec>::T;
    constexpr int kWidth = 32 * kK;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int local = static_cast<int>(blockIdx.x) * static_cast<int>(blockDim.x >> 5) + warp;
    if (local >= a.count) return;
    const int w = a.first + local;
    Control* ctl = v.ctl;
    if (a.epoch_mode && *reinterpret_cast<volatile int32_t*>(&ctl->done)) return;

    const CsrSweepLayout L = csr_sweep_layout(v.max_window_bins, kWidth, sizeof(VT), kCollect);
    const CsrSlot S = csr_slot(kWidth, sizeof(VT));
    unsigned char* base = smem + static_cast<size_t>(warp) * L.total;
    unsigned char* ring = base + L.slots;
    const uint32_t ring_addr = static_cast<uint32_t>(__cvta_generic_to_shared(ring));
    double* lg_s = reinterpret_cast<double*>(base + L.log_g);
    uint64_t* h_s = reinterpret_cast<uint64_t*>(base + L.hist);
    uint32_t* hd = reinterpret_cast<uint32_t*>(base + L.hd);
    uint8_t* act_s = base + L.active;
    double* sq_s = reinterpret_cast<double*>(base + L.sq);
    uint64_t* ds_s = reinterpret_cast<uint64_t*>(base + L.ds);

    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window], nbins = we - wb;
    if (st.cur_bin < wb || st.cur_bin >= we) {  // "Walker escaped its energy window"
        if (lane == 0) record_error(ctl, WLG_ERR_ESCAPED, w);
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
    double* fg = v.fields + static_cast<size_t>(st.slot) * v.ld;
    int8_t* sg = v.spins + static_cast<size_t>(st.slot) * v.ld;
    const int32_t* __restrict__ ecol = v.ell_col;
    const VT* __restrict__ evals = ell_values<kPrec>(v);
    const FastMod fm = v.site_mod;

    for (int b = lane; b < nbins; b += 32) {
        lg_s[b] = v.log_g[boff + b];
        h_s[b] = v.hist[boff + b];
        act_s[b] = v.active[boff + b];
        hd[b] = 0;
        if constexpr (kCollect) {
            sq_s[b] = v.sqdisp[boff + b];
            ds_s[b] = v.dsamples[boff + b];
        }
    }
    __syncwarp();
    // pilot statistics (src/wang_landau.cpp:272-276, 317-342): round trips and representatives
    const double lower = window_lower(v, wb), upper = window_lower(v, we);
    int32_t rt_state = st.rt_state;
    uint64_t trips = st.round_trips;
    if (kCollect && st.rep_pending) {  // a replica exchange changed the configuration
        warp_update_representatives(v, w, st.energy, sg, lane);
        st.rep_pending = 0;
    }

    auto site_of = [&](uint64_t d) -> int { return d < fm.threshold ? -1 : static_cast<int>(fast_mod(fm, d)); };
    auto slot_ptr = [&](int k) { return ring + static_cast<size_t>(k & (kCsrSlots - 1)) * S.bytes; };
    auto slot_addr = [&](int k) { return ring_addr + static_cast<uint32_t>((k & (kCsrSlots - 1)) * S.bytes); };
    // copy one site's row, field and spin word into ring slot k (one commit group)
    auto fetch = [&](int k, int site) {
        const int s = site < 0 ? 0 : site;
        const uint32_t dst = slot_addr(k);
        const unsigned char* crow = reinterpret_cast<const unsigned char*>(ecol + static_cast<size_t>(s) * kWidth);
        const unsigned char* vrow = reinterpret_cast<const unsigned char*>(evals + static_cast<size_t>(s) * kWidth);
#pragma unroll
        for (int c = lane; c < kWidth * 4 / 16; c += 32) cp_async16(dst + static_cast<uint32_t>(S.col + 16 * c), crow + 16 * c);
#pragma unroll
        for (int c = lane; c < kWidth * static_cast<int>(sizeof(VT)) / 16; c += 32)
            cp_async16(dst + static_cast<uint32_t>(S.val + 16 * c), vrow + 16 * c);
        if (lane == 0) cp_async8(dst + static_cast<uint32_t>(S.f), fg + s);
        if (lane == 1) cp_async4(dst + static_cast<uint32_t>(S.sword), sg + (s & ~3));
        cp_commit();
    };
    // copy the neighbour fields of the site in slot k (lane j: entries j, j+32, ...; one group)
    auto load_neighbours = [&](int k) {
        const unsigned char* p = slot_ptr(k);
        const uint32_t dst = slot_addr(k);
#pragma unroll
        for (int e = 0; e < kK; ++e) {
            const int c = reinterpret_cast<const int32_t*>(p + S.col)[lane + 32 * e];
            if (c >= 0) cp_async8(dst + static_cast<uint32_t>(S.nf + 8 * (lane + 32 * e)), fg + c);
        }
        cp_commit();
    };
    auto slot_field = [&](int k) -> double& { return *reinterpret_cast<double*>(slot_ptr(k) + S.f); };
    auto slot_spin = [&](int k, int site) -> int {
        const uint32_t word = *reinterpret_cast<const uint32_t*>(slot_ptr(k) + S.sword);
        return static_cast<int8_t>(static_cast<uint8_t>(word >> (8 * (site & 3))));
    };
    // the candidate `site` in slot k after the accepted flip of `flipped` (slot kf), factor m;
    // every copy has landed
    auto correct = [&](int k, int site, int kf, int flipped, double m) {
        const unsigned char* pf = slot_ptr(kf);
        bool hit = false;
        double jv = 0.0;
#pragma unroll
        for (int e = 0; e < kK; ++e)
            if (site >= 0 && reinterpret_cast<const int32_t*>(pf + S.col)[lane + 32 * e] == site) {
                hit = true;
                jv = static_cast<double>(reinterpret_cast<const VT*>(pf + S.val)[lane + 32 * e]);
            }
        const unsigned mask = __ballot_sync(kFull, hit);
        if (mask) {
            jv = __shfl_sync(kFull, jv, __ffs(mask) - 1);
            if (lane == 0) slot_field(k) = fma(m, jv, slot_field(k));
        }
        if (site == flipped && lane == 1)  // the spin byte: +1 (0x01) <-> -1 (0xff)
            *reinterpret_cast<uint32_t*>(slot_ptr(k) + S.sword) ^= 0xfeu << (8 * (site & 3));
    };

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
    uint64_t active_before = 0;
    if (stage != kInverseTime) {
        for (int b = lane; b < nbins; b += 32) active_before += act_s[b] ? 1 : 0;
        active_before = warp_sum_u64(active_before);
    }

    // Slots o, o+1, o+2 (mod 4) hold the site of the next attempt (draw hq) and the candidates
    // (draws hq+1, hq+2); site indices i0, i1, i2.
    // The draws come in batches of 32: every lane steps the generator through the batch and
    // keeps draw j = lane, with its site and log(max(u, 2^-53)) (src/wang_landau.cpp:250, 261);
    // an attempt reads them from the owning lane.  Two batches are held: draws [first, first+64).
    Rng rng{st.rng[0], st.rng[1], st.rng[2], st.rng[3]};
    auto generate = [&](int& site, double& log_u) {
        uint64_t mine = 0;
#pragma unroll 4
        for (int j = 0; j < 32; ++j) {
            const uint64_t d = rng.next();
            mine = lane == j ? d : mine;
        }
        site = site_of(mine);
        log_u = log(fmax(to_uniform(mine), 0x1.0p-53));
    };
    uint32_t first = 0, hq = 0;  // draw index of lane 0 of the first batch; of the current site
    int site_a, site_b;
    double lnu_a, lnu_b;
    generate(site_a, lnu_a);
    generate(site_b, lnu_b);
    auto draw_site = [&](uint32_t k) { return __shfl_sync(kFull, k < first + 32 ? site_a : site_b, k & 31); };
    auto draw_lnu = [&](uint32_t k) { return __shfl_sync(kFull, k < first + 32 ? lnu_a : lnu_b, k & 31); };
    int o = 0;
    int i0 = draw_site(0), i1 = draw_site(1), i2 = draw_site(2);
    fetch(0, i0);
    fetch(1, i1);
    fetch(2, i2);
    cp_wait<0>();
    __syncwarp();
    load_neighbours(0);
    double lnu = draw_lnu(1);
    // after the site moved to draw hq: keep hq+4 inside the two batches
    auto advance_batches = [&]() {
        if (hq >= first + 32) {
            site_a = site_b;
            lnu_a = lnu_b;
            first += 32;
            generate(site_b, lnu_b);
        }
    };

    // The attempts of one batch; kIT selects the 1/t stage (per-attempt factor and active
    // count) or the Wang-Landau / frozen stages (constant factor).
    auto run = [&](auto it_tag) {
        constexpr bool kIT = decltype(it_tag)::value;
        const bool frozen = stage == kFrozen;
        InverseTimeTable itt;  // the 1/t factors of the coming attempts
        // 1/t stage: an attempt's factor and freeze are applied to log g of its bin at the point
        // where the next attempt first reads log g, so the factor's shuffle is not waited for
        double lg_base_p = 0.0, f_p = 0.0;
        bool pend = false;
        for (uint32_t t = 0; t < batch;) {
            if (i0 < 0) {  // rare: bounded() rejects draw hq; the next draw is the site
                hq += 1;
                advance_batches();
                i0 = i1;
                i1 = i2;
                i2 = draw_site(hq + 2);
                fetch(o + 3, i2);
                o = (o + 1) & (kCsrSlots - 1);
                cp_wait<2>();  // the new site's row (an older group) has landed
                __syncwarp();
                load_neighbours(o);
                lnu = draw_lnu(hq + 1);
                continue;
            }
            // the decision (attempt_flip, src/wang_landau.cpp:244-262)
            const int si = slot_spin(o, i0);
            const double m = si > 0 ? -2.0 : 2.0;  // -2 * spin
            const double Ep = fma(m, slot_field(o), E);
            const bool in_range = Ep >= g.minimum && Ep <= g.maximum;
            const double qv = kPow2 ? fma(Ep, g.inv_width, neg_min_scaled) : (Ep - g.minimum) / g.width;
            int nb = in_range ? bin_floor(qv) : -1;
            nb = (nb == gcount && Ep == g.maximum) ? gcount - 1 : nb;
            const bool in_window = nb >= wb && nb < we;
            const double lg_load = lg_s[in_window ? nb - wb : 0];
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
            const bool forced = !det && since >= force_limit;
            const bool need_u = in_window && !det && !forced;
            const bool accepted = in_window && (det || forced || lnu < log_ratio);

            if (accepted) {  // add_flip_delta, and the candidates brought up to date
                cp_wait<0>();
                __syncwarp();
                const unsigned char* ps = slot_ptr(o);
#pragma unroll
                for (int e = 0; e < kK; ++e) {
                    const int j = lane + 32 * e;
                    const int c = reinterpret_cast<const int32_t*>(ps + S.col)[j];
                    if (c >= 0)
                        fg[c] = fma(m, static_cast<double>(reinterpret_cast<const VT*>(ps + S.val)[j]),
                                    reinterpret_cast<const double*>(ps + S.nf)[j]);
                }
                if (lane == 0) sg[i0] = static_cast<int8_t>(-si);
                correct(o + 2, i2, o, i0, m);
                if (!need_u) correct(o + 1, i1, o, i0, m);  // draw hq+1 becomes the next site
            }
            E = accepted ? Ep : E;
            since = accepted ? 0 : since + 1;
            n_acc += accepted ? 1u : 0u;
            n_forced += (accepted && forced) ? 1u : 0u;
            ++t;
            if (kCollect && lane == 0) {  // the displacement out of the old bin, 0 when rejected
                const double displacement = accepted ? m * slot_field(o) : 0.0;
                sq_s[cur - wb] += displacement * displacement;
                ++ds_s[cur - wb];
            }

            // update_inverse_time_factor then update_current_bin (src/wang_landau.cpp:277-278)
            if (kIT && stage == kInverseTime) {  // resolved at the next read of log g
                f_p = inverse_time_factor(itt, att0 + st.time_offset + t - 1, active_count, factor, lane);
                pend = true;
            }
            const bool move = accepted && nb != cur;
            const int ncur = move ? nb : cur;
            const double lg_base = move ? lg_new : lg_cur;
            if (kIT) {
                const bool visited = act_s[ncur - wb] != 0;
                active_count += visited ? 0 : 1;
            }
            if (lane == 0) {
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

            __syncwarp();  // this attempt's stores and reads of the slots precede later copies
            if (kCollect && accepted) {
                round_trip_update(E, lower, upper, P.round_trip_margin, rt_state, trips);
                warp_update_representatives(v, w, E, sg, lane);
            }
            if (need_u) {  // draw hq+1 was the uniform: the site is draw hq+2
                hq += 2;
                advance_batches();
                i0 = i2;
                i1 = draw_site(hq + 1);
                i2 = draw_site(hq + 2);
                fetch(o + 3, i1);
                fetch(o + 4, i2);  // the slot of the site just done
                o = (o + 2) & (kCsrSlots - 1);
                cp_wait<3>();  // the new site's row (older than the last three groups) has landed
            } else {
                hq += 1;
                advance_batches();
                i0 = i1;
                i1 = i2;
                i2 = draw_site(hq + 2);
                fetch(o + 3, i2);
                o = (o + 1) & (kCsrSlots - 1);
                cp_wait<2>();
            }
            __syncwarp();
            load_neighbours(o);
            lnu = draw_lnu(hq + 1);
        }
        if (kIT && pend) {  // the last attempt's factor
            const bool frz = f_p <= P.final_factor;
            stage = frz ? kFrozen : stage;
            factor = f_p;
            lg_cur = frz ? lg_base_p : lg_base_p + f_p;
        }
    };
    if (stage == kInverseTime)
        run(std::true_type{});
    else
        run(std::false_type{});
    cp_wait<0>();  // no copy is in flight when the walker leaves

    // the generator is at draw first+64; step back to the last consumed draw, hq-1
    for (uint32_t k = hq; k != first + 64; ++k) rng_step_back(rng);
    if (lane == 0) lg_s[cur - wb] = lg_cur;
    __syncwarp();
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
    st.rt_state = rt_state;
    st.round_trips = trips;

    if (a.epoch_mode && st.stage == kWangLandau) {
        const bool at_limit = P.max_attempts != 0 && st.attempted >= P.max_attempts;
        if (st.attempted - st.last_check >= P.check_interval || at_limit) {
            st.last_check = st.attempted;
            const HistStats hs = warp_histogram_statistics(h_s, act_s, nbins, st.active_count, lane);
            st.last_flatness = P.inverse_time ? hs.coverage : hs.min_over_mean;
            if (stats_ready(hs, st.stage, P)) warp_begin_next_iteration(st, h_s, nullptr, nbins, P, lane);
        }
    }
    for (int b = lane; b < nbins; b += 32) {
        v.log_g[boff + b] = lg_s[b];
        v.hist[boff + b] = h_s[b];
        v.active[boff + b] = act_s[b];
        if constexpr (kCollect) {
            v.sqdisp[boff + b] = sq_s[b];
            v.dsamples[boff + b] = ds_s[b];
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

using SweepFn = void (*)(EngineView, WalkArgs);

template <int kK, bool kPow2, int kPrec, bool kCollect>
SweepFn csr_fn() {
    static bool configured = false;
    if (!configured) {
        check_cuda(cudaFuncSetAttribute(reinterpret_cast<const void*>(&sweep_csr_kernel<kK, kPow2, kPrec, kCollect>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    return &sweep_csr_kernel<kK, kPow2, kPrec, kCollect>;
}

template <bool kPow2, int kPrec, bool kCollect>
SweepFn pick_csr_width(int width) {
    switch (width) {
        case 32: return csr_fn<1, kPow2, kPrec, kCollect>();
        case 64: return csr_fn<2, kPow2, kPrec, kCollect>();
        case 128: return csr_fn<4, kPow2, kPrec, kCollect>();
        case 256: return csr_fn<8, kPow2, kPrec, kCollect>();
        default: return nullptr;
    }
}

template <bool kCollect>
SweepFn pick_csr(const EngineView& v) {
    const bool pow2 = v.grid.pow2_width != 0;
    if (v.precision == WLG_PRECISION_FP32)
        return pow2 ? pick_csr_width<true, WLG_PRECISION_FP32, kCollect>(v.ell_width)
                    : pick_csr_width<false, WLG_PRECISION_FP32, kCollect>(v.ell_width);
    return pow2 ? pick_csr_width<true, WLG_PRECISION_FP64, kCollect>(v.ell_width)
                : pick_csr_width<false, WLG_PRECISION_FP64, kCollect>(v.ell_width);
}

}  // namespace

namespace {

// ELLPACK copy of the CSR couplings: one warp per row, entries [0, row length) from the CSR
// row in column order, then column -1 / value 0 up to `width`.
__global__ void ell_fill_kernel(int n, int width, const int32_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                const double* __restrict__ val64, const float* __restrict__ val32,
                                int32_t* __restrict__ ell_col, double* __restrict__ ell_val64,
                                float* __restrict__ ell_val32) {
    const int lane = threadIdx.x & 31;
    const int row = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (row >= n) return;
    const int begin = ptr[row], count = ptr[row + 1] - begin;
    for (int e = lane; e < width; e += 32) {
        const size_t at = static_cast<size_t>(row) * width + e;
        const bool in = e < count;
        ell_col[at] = in ? col[begin + e] : -1;
        if (ell_val64) ell_val64[at] = in ? val64[begin + e] : 0.0;
        if (ell_val32) ell_val32[at] = in ? val32[begin + e] : 0.0f;
    }
}

}  // namespace

void launch_ell_fill(int n, int width, const int32_t* ptr, const int32_t* col, const double* val64,
                     const float* val32, int32_t* ell_col, double* ell_val64, float* ell_val32, cudaStream_t stream) {
    if (n <= 0) return;
    const unsigned blocks = static_cast<unsigned>((n + 7) / 8);
    ell_fill_kernel<<<blocks, 256, 0, stream>>>(n, width, ptr, col, val64, val32, ell_col, ell_val64, ell_val32);
    check_cuda(cudaGetLastError(), "ell_fill_kernel");
}

bool launch_sweep_csr(const EngineView& v, const WalkArgs& a, int walkers_per_block, cudaStream_t stream) {
    if (!v.csr || v.ell_width == 0 || v.p.nalivaiko) return false;  // the Nalivaiko mask: walk_kernel
    const bool collect = v.p.collect != 0;
    SweepFn fn = collect ? pick_csr<true>(v) : pick_csr<false>(v);
    if (!fn) return false;
    const int vbytes = v.precision == WLG_PRECISION_FP32 ? 4 : 8;
    const size_t per_walker = csr_sweep_layout(v.max_window_bins, v.ell_width, vbytes, collect).total;
    if (per_walker > 227 * 1024) return false;
    int wpb = walkers_per_block < 1 ? 1 : (walkers_per_block > 8 ? 8 : walkers_per_block);
    while (wpb > 1 && per_walker * static_cast<size_t>(wpb) > 227 * 1024) --wpb;
    const unsigned blocks = static_cast<unsigned>((a.count + wpb - 1) / wpb);
    fn<<<blocks, 32 * wpb, per_walker * static_cast<size_t>(wpb), stream>>>(v, a);
    check_cuda(cudaGetLastError(), "sweep_csr_kernel");
    return true;
}

}  // namespace wlg
