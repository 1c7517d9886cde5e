// rewl.cu — the replica-exchange step, the end-of-run summaries and single-walker ops.
//
//  * exchange_kernel: the even/odd exchange of run_rewl (src/parallel.cpp:410-421) with
//    local_exchange (src/parallel.cpp:157-166), exchange_log_probability and
//    swap_configuration (src/wang_landau.cpp:483-508).  All pairs of one parity are
//    independent (the pairing p -> (p+epoch) % pairs is a permutation and the boundaries of
//    one parity are disjoint), so one thread handles one pair.  A swap exchanges the two
//    walkers' configuration slots, energies and bins; no spin or field is copied.  One CTA
//    also closes the epoch: termination test (all frozen, or all at the attempt limit,
//    src/parallel.cpp:527-533) and the epoch counter.
//  * summarize_kernel: summarize_impl (src/parallel.cpp:23-62).
//  * sampling_kernel: summarize_sampling_impl (src/parallel.cpp:64-78).
//  * statistics_kernel: the per-walker statistics of run_rewl (src/parallel.cpp:541-553).
#include <cmath>

#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

__device__ __forceinline__ int32_t wbegin(const EngineView& v, int w) { return v.win_begin[v.ws[w].window]; }
__device__ __forceinline__ int32_t wend(const EngineView& v, int w) { return v.win_end[v.ws[w].window]; }

// exchange_log_probability (src/wang_landau.cpp:497-508)
__device__ double exchange_log_probability(const EngineView& v, int L, int R) {
    const WalkerState& a = v.ws[L];
    const WalkerState& b = v.ws[R];
    const int ab = wbegin(v, L), ae = wend(v, L), bb = wbegin(v, R), be = wend(v, R);
    const int x = a.cur_bin, y = b.cur_bin;
    const bool valid = x >= ab && x < ae && y >= ab && y < ae && x >= bb && x < be && y >= bb && y < be;
    if (!valid) return -INFINITY;
    const size_t bins = static_cast<size_t>(v.grid.count);
    const double* ga = v.log_g + static_cast<size_t>(L) * bins;
    const double* gb = v.log_g + static_cast<size_t>(R) * bins;
    return ga[x] - ga[y] + gb[y] - gb[x];
}

// swap_configuration (src/wang_landau.cpp:483-495) without moving data: slots, energies
// and bins are exchanged; the representative bank is refreshed by the next sweep.
__device__ void swap_configuration(const EngineView& v, int L, int R) {
    WalkerState& a = v.ws[L];
    WalkerState& b = v.ws[R];
    const int32_t slot = a.slot;
    a.slot = b.slot;
    b.slot = slot;
    const double e = a.energy;
    a.energy = b.energy;
    b.energy = e;
    const int32_t bin = a.cur_bin;
    a.cur_bin = b.cur_bin;
    b.cur_bin = bin;
    if (v.p.collect) {
        round_trip_update(a.energy, window_lower(v, wbegin(v, L)), window_lower(v, wend(v, L)),
                          v.p.round_trip_margin, a.rt_state, a.round_trips);
        round_trip_update(b.energy, window_lower(v, wbegin(v, R)), window_lower(v, wend(v, R)),
                          v.p.round_trip_margin, b.rt_state, b.round_trips);
        a.rep_pending = 1;
        b.rep_pending = 1;
    }
}

__global__ void exchange_kernel(EngineView v) {
    __shared__ uint64_t s_epoch;
    __shared__ int s_skip;
    __shared__ unsigned s_accepted;
    Control* c = v.ctl;
    if (threadIdx.x == 0) {
        s_skip = c->done;
        s_epoch = c->epoch;
        s_accepted = 0;
    }
    __syncthreads();
    if (s_skip) return;
    const uint64_t epoch = s_epoch;
    const int parity = static_cast<int>(epoch & 1ULL);
    const int wpw = v.walkers_per_window;
    const int nbound = v.windows - 2 < parity ? 0 : (v.windows - 2 - parity) / 2 + 1;
    const int npairs = nbound * wpw;
    for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
        const int k = t / wpw, p = t % wpw;
        const int b = parity + 2 * k;
        const int L = b * wpw + p;
        const int R = (b + 1) * wpw + static_cast<int>((static_cast<uint64_t>(p) + epoch) % static_cast<uint64_t>(wpw));
        const double logp = exchange_log_probability(v, L, R);
        bool accept = false;
        if (isfinite(logp)) {
            if (logp >= 0.0) {
                accept = true;
            } else {
                Rng rng;
                rng.seed(v.p.seed ^ (epoch * 0x9e3779b97f4a7c15ULL), static_cast<uint64_t>(b));
                accept = log(fmax(to_uniform(rng.next()), 0x1.0p-53)) < logp;
            }
        }
        if (accept) {
            swap_configuration(v, L, R);
            atomicAdd(&s_accepted, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        c->exchange_attempted += static_cast<uint64_t>(npairs);
        c->exchange_accepted += s_accepted;
        const bool all_frozen = c->frozen == static_cast<uint32_t>(v.walkers);
        const bool limit = v.p.max_attempts != 0 && c->at_limit == static_cast<uint32_t>(v.walkers);
        c->done = (all_frozen || limit || c->error != 0) ? 1 : 0;
        c->frozen = 0;
        c->at_limit = 0;
        c->epoch = epoch + 1;
    }
}

// Applies representative updates left pending by exchanges (one warp per walker).
__global__ void flush_pending_kernel(EngineView v) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= v.walkers) return;
    WalkerState& st = v.ws[w];
    if (!v.p.collect || !st.rep_pending) return;
    const int8_t* s = v.spins + static_cast<size_t>(st.slot) * v.ld;
    warp_update_representatives(v, w, st.energy, s, lane);
    if (lane == 0) st.rep_pending = 0;
}

// summarize_impl for one window; status 1 = "no common active bin".
// One CTA per window: window0 + blockIdx.x, whose outputs (bins entries each) and status are
// at offset blockIdx.x.
__global__ void summarize_kernel(EngineView v, int window0, int allow_empty, double* log_g, uint64_t* hist,
                                 double* sem, uint8_t* valid, int* status) {
    const int window = window0 + static_cast<int>(blockIdx.x);
    const int wb = v.win_begin[window], we = v.win_end[window];
    const int first = window * v.walkers_per_window, count = v.walkers_per_window;
    const size_t bins = static_cast<size_t>(v.grid.count);
    log_g += blockIdx.x * bins;
    hist += blockIdx.x * bins;
    sem += blockIdx.x * bins;
    valid += blockIdx.x * bins;
    status += blockIdx.x;
    __shared__ int s_ref;
    if (threadIdx.x == 0) s_ref = we;
    for (size_t i = threadIdx.x; i < bins; i += blockDim.x) {
        log_g[i] = NAN;
        hist[i] = 0;
        sem[i] = NAN;
        valid[i] = 0;
    }
    __syncthreads();
    for (int i = wb + threadIdx.x; i < we; i += blockDim.x) {
        bool ok = true;
        uint64_t h = 0;
        for (int k = 0; k < count; ++k) {
            const size_t at = static_cast<size_t>(first + k) * bins + i;
            ok = ok && v.active[at] != 0;
            h += v.hist[at];
        }
        valid[i] = ok ? 1 : 0;
        hist[i] = h;
        if (ok) atomicMin(&s_ref, i);
    }
    __syncthreads();
    const int ref = s_ref;
    if (ref == we) {
        if (threadIdx.x == 0) *status = allow_empty ? 0 : 1;
        return;
    }
    for (int i = wb + threadIdx.x; i < we; i += blockDim.x) {
        if (!valid[i]) continue;
        double mean = 0.0;
        for (int k = 0; k < count; ++k) {
            const double* g = v.log_g + static_cast<size_t>(first + k) * bins;
            mean += g[i] - g[ref];
        }
        mean /= static_cast<double>(count);
        log_g[i] = mean;
        if (count > 1) {
            double sd = 0.0;
            for (int k = 0; k < count; ++k) {
                const double* g = v.log_g + static_cast<size_t>(first + k) * bins;
                const double value = g[i] - g[ref];
                const double delta = value - mean;
                sd += delta * delta;
            }
            sem[i] = sqrt(sd / (static_cast<double>(count) * static_cast<double>(count - 1)));
        }
    }
    if (threadIdx.x == 0) *status = 0;
}

// summarize_sampling_impl (src/parallel.cpp:64-78) for one window.
__global__ void sampling_kernel(EngineView v, int window, double* sq, uint64_t* samples, uint64_t* trips) {
    const int wb = v.win_begin[window], we = v.win_end[window];
    const int first = window * v.walkers_per_window, count = v.walkers_per_window;
    const size_t bins = static_cast<size_t>(v.grid.count);
    for (size_t i = threadIdx.x; i < bins; i += blockDim.x) {
        double s = 0.0;
        uint64_t d = 0;
        if (static_cast<int>(i) >= wb && static_cast<int>(i) < we)
            for (int k = 0; k < count; ++k) {
                s += v.sqdisp[static_cast<size_t>(first + k) * bins + i];
                d += v.dsamples[static_cast<size_t>(first + k) * bins + i];
            }
        sq[i] = s;
        samples[i] = d;
    }
    if (threadIdx.x == 0) {
        uint64_t t = 0;
        for (int k = 0; k < count; ++k) t += v.ws[first + k].round_trips;
        *trips = t;
    }
}

// One warp per walker: the WalkerStatistics row of run_rewl.
__global__ void statistics_kernel(EngineView v, wlg_walker_statistics* out) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= v.walkers) return;
    const WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window];
    const size_t off = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + wb;
    const uint8_t* mask = v.p.nalivaiko ? v.refine + off : v.active + off;
    const HistStats hs = warp_histogram_statistics(v.hist + off, mask, we - wb,
                                                   v.p.nalivaiko ? st.refine_count : st.active_count, lane);
    if (lane == 0) {
        wlg_walker_statistics r;
        r.walker_id = static_cast<uint64_t>(w);
        r.window_id = static_cast<uint64_t>(st.window);
        r.mpi_rank = 0;
        r.attempted = st.attempted;
        r.accepted = st.accepted;
        r.forced_accepted = st.forced;
        r.attempts_since_last_accepted = st.attempted - st.last_accepted;
        r.energy = st.energy;
        r.factor = st.factor;
        r.active_bins = hs.active_bins;
        r.minimum_histogram = hs.minimum;
        r.mean_histogram = hs.mean;
        r.min_over_mean = hs.min_over_mean;
        r.round_trips = st.round_trips;
        out[w] = r;
    }
}

// Single-walker histogram statistics + flat/covered/ready flags.
__global__ void walker_stats_kernel(EngineView v, int w, wlg_histogram_statistics* out, int* flags) {
    const int lane = threadIdx.x & 31;
    const WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window];
    const size_t off = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + wb;
    const uint8_t* mask = v.p.nalivaiko ? v.refine + off : v.active + off;
    const HistStats hs = warp_histogram_statistics(v.hist + off, mask, we - wb,
                                                   v.p.nalivaiko ? st.refine_count : st.active_count, lane);
    if (lane == 0) {
        out->active_bins = hs.active_bins;
        out->covered_bins = hs.covered;
        out->minimum = hs.minimum;
        out->mean = hs.mean;
        out->min_over_mean = hs.min_over_mean;
        out->coverage = hs.coverage;
        flags[0] = stats_flat(hs, st.stage, v.p) ? 1 : 0;
        flags[1] = stats_covered(hs, st.stage) ? 1 : 0;
        flags[2] = stats_ready(hs, st.stage, v.p) ? 1 : 0;
    }
}

// begin_next_iteration on one walker; status 1 = "WL iteration is not complete".
__global__ void begin_iteration_kernel(EngineView v, int w, int* status) {
    const int lane = threadIdx.x & 31;
    WalkerState st = v.ws[w];
    const int wb = v.win_begin[st.window], we = v.win_end[st.window];
    const size_t off = static_cast<size_t>(w) * static_cast<size_t>(v.grid.count) + wb;
    const uint8_t* mask = v.p.nalivaiko ? v.refine + off : v.active + off;
    const HistStats hs = warp_histogram_statistics(v.hist + off, mask, we - wb,
                                                   v.p.nalivaiko ? st.refine_count : st.active_count, lane);
    if (!stats_ready(hs, st.stage, v.p)) {
        if (lane == 0) *status = 1;
        return;
    }
    warp_begin_next_iteration(st, v.hist + off, v.refine + off, we - wb, v.p, lane);
    if (lane == 0) {
        v.ws[w] = st;
        *status = 0;
    }
}

// exchange_log_probability and, when do_swap, swap_configuration for one pair (a warp, so
// that the representative refresh can run).  status 1 = "would violate an energy window".
__global__ void exchange_pair_kernel(EngineView v, int L, int R, int do_swap, double* logp, int* status) {
    const int lane = threadIdx.x & 31;
    const double lp = exchange_log_probability(v, L, R);
    if (lane == 0) *logp = lp;
    if (!do_swap) return;
    const WalkerState& a = v.ws[L];
    const WalkerState& b = v.ws[R];
    const int this_bin = b.cur_bin, other_bin = a.cur_bin;
    const bool ok = this_bin >= wbegin(v, L) && this_bin < wend(v, L) && other_bin >= wbegin(v, R) &&
                    other_bin < wend(v, R);
    __syncwarp();
    if (!ok) {
        if (lane == 0) *status = 1;
        return;
    }
    if (lane == 0) swap_configuration(v, L, R);
    __syncwarp();
    if (v.p.collect) {
        for (int k = 0; k < 2; ++k) {
            const int w = k == 0 ? L : R;
            WalkerState& st = v.ws[w];
            warp_update_representatives(v, w, st.energy, v.spins + static_cast<size_t>(st.slot) * v.ld, lane);
            __syncwarp();
            if (lane == 0) st.rep_pending = 0;
            __syncwarp();
        }
    }
    if (lane == 0) *status = 0;
}

// ---- launchers ------------------------------------------------------------------------------

void launch_exchange(const EngineView& v, cudaStream_t stream) {
    exchange_kernel<<<1, 256, 0, stream>>>(v);
    check_cuda(cudaGetLastError(), "exchange_kernel");
}

void launch_flush_pending(const EngineView& v, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((v.walkers * 32 + 255) / 256);
    flush_pending_kernel<<<blocks, 256, 0, stream>>>(v);
    check_cuda(cudaGetLastError(), "flush_pending_kernel");
}

void launch_summarize(const EngineView& v, int window, int windows, int allow_empty, double* log_g, uint64_t* hist,
                      double* sem, uint8_t* valid, int* status, cudaStream_t stream) {
    summarize_kernel<<<static_cast<unsigned>(windows), 256, 0, stream>>>(v, window, allow_empty, log_g, hist, sem, valid,
                                                                         status);
    check_cuda(cudaGetLastError(), "summarize_kernel");
}

void launch_sampling(const EngineView& v, int window, double* sq, uint64_t* samples, uint64_t* trips,
                     cudaStream_t stream) {
    sampling_kernel<<<1, 256, 0, stream>>>(v, window, sq, samples, trips);
    check_cuda(cudaGetLastError(), "sampling_kernel");
}

void launch_walker_statistics(const EngineView& v, wlg_walker_statistics* out, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((v.walkers * 32 + 255) / 256);
    statistics_kernel<<<blocks, 256, 0, stream>>>(v, out);
    check_cuda(cudaGetLastError(), "statistics_kernel");
}

void launch_histogram_statistics(const EngineView& v, int walker, wlg_histogram_statistics* out, int* flags,
                                 cudaStream_t stream) {
    walker_stats_kernel<<<1, 32, 0, stream>>>(v, walker, out, flags);
    check_cuda(cudaGetLastError(), "walker_stats_kernel");
}

void launch_begin_next_iteration(const EngineView& v, int walker, int* status, cudaStream_t stream) {
    begin_iteration_kernel<<<1, 32, 0, stream>>>(v, walker, status);
    check_cuda(cudaGetLastError(), "begin_iteration_kernel");
}

void launch_exchange_pair(const EngineView& v, int left, int right, int do_swap, double* logp, int* status,
                          cudaStream_t stream) {
    exchange_pair_kernel<<<1, 32, 0, stream>>>(v, left, right, do_swap, logp, status);
    check_cuda(cudaGetLastError(), "exchange_pair_kernel");
}

}  // namespace wlg
