// stitch.cu — stitch_dos (src/analysis.cpp:45-130) on the device, straight from the
// fragments summarize_kernel leaves in device memory: the run's density of states comes back
// in one copy instead of windows x bins.
//
// One CTA.  The joins are sequential (the left curve of join f holds the shifted values of
// join f-1), the work inside a join is parallel over the overlap's bins:
//   * the fallback join, the common valid bin nearest the overlap's midpoint, and the slope
//     join, the bin where the two curves' five-point least-squares slopes agree best, are
//     arg-min reductions over (key, bin) pairs, so ties go to the lowest bin, as the
//     reference's ascending loops with a strict < give them;
//   * every slope is one thread's sequential sum over its five bins in ascending order, the
//     reference's operation order, so each key is bit-identical to the host's;
//   * the join quality (an addition: common bins, RMSE, maximum deviation, slope mismatch) is
//     summed by one thread in bin order, as the host version does.
// The peak normalisation (a maximum and a subtraction) is done here; the complete-range
// normalisation needs exp and log of the C library to match the reference bit for bit, so the
// host adds that one constant after the copy.
#include <cmath>

#include "engine.hpp"

namespace wlg {

namespace {

constexpr int kStitchThreads = 256;

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

// local_slope (src/analysis.cpp:22-40): least-squares slope of the valid, finite bins among
// centre-2 .. centre+2 clipped to [begin, end), per unit energy; NaN below two points.
__device__ double slope_at(const double* lg, const uint8_t* ok, int centre, int begin, int end, double width) {
    const int lo = centre > 2 ? max(begin, centre - 2) : begin;
    const int hi = min(end, centre + 3);
    int points = 0;
    double sx = 0.0, sy = 0.0;
    for (int i = lo; i < hi; ++i)
        if (ok[i] != 0 && finite(lg[i])) {
            sx += static_cast<double>(i);
            sy += lg[i];
            ++points;
        }
    if (points < 2) return nan("");
    sx /= static_cast<double>(points);
    sy /= static_cast<double>(points);
    double sxy = 0.0, sxx = 0.0;
    for (int i = lo; i < hi; ++i)
        if (ok[i] != 0 && finite(lg[i])) {
            const double dx = static_cast<double>(i) - sx;
            sxy += dx * (lg[i] - sy);
            sxx += dx * dx;
        }
    return sxx > 0.0 ? sxy / sxx / width : nan("");
}

// Block arg-min of (key, bin): the smallest key, the lowest bin among equal keys.  Threads
// without a candidate pass key = +inf and bin = INT_MAX.
__device__ void argmin(double& key, int& bin, double* s_key, int* s_bin) {
    for (int o = 16; o > 0; o >>= 1) {
        const double k2 = __shfl_down_sync(0xffffffffu, key, o);
        const int b2 = __shfl_down_sync(0xffffffffu, bin, o);
        if (k2 < key || (k2 == key && b2 < bin)) {
            key = k2;
            bin = b2;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        s_key[warp] = key;
        s_bin[warp] = bin;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kStitchThreads / 32; ++w)
            if (s_key[w] < s_key[0] || (s_key[w] == s_key[0] && s_bin[w] < s_bin[0])) {
                s_key[0] = s_key[w];
                s_bin[0] = s_bin[w];
            }
    }
    __syncthreads();
    key = s_key[0];
    bin = s_bin[0];
}

__global__ void __launch_bounds__(kStitchThreads) stitch_kernel(int windows, int bins, const int32_t* wbeg,
                                                                const int32_t* wend, const double* flg,
                                                                const uint64_t* fh, const double* fse,
                                                                const uint8_t* fv, const int* summarize_status,
                                                                double width, int complete_range, double* lg,
                                                                uint64_t* h, double* se, uint8_t* ok,
                                                                wlg_join_quality* joins, int* status) {
    __shared__ double s_key[kStitchThreads / 32];
    __shared__ int s_bin[kStitchThreads / 32];
    __shared__ int s_err;
    const int t = static_cast<int>(threadIdx.x);
    if (t == 0) {
        s_err = 0;
        for (int w = 0; w < windows; ++w)
            if (summarize_status[w] != 0) s_err = kStitchNoCommonBin;
    }
    __syncthreads();
    if (s_err != 0) {
        if (t == 0) *status = s_err;
        return;
    }
    const double qnan = nan("");
    for (int i = t; i < bins; i += kStitchThreads) {
        lg[i] = qnan;
        se[i] = qnan;
        h[i] = 0;
        ok[i] = 0;
    }
    __syncthreads();
    for (int i = wbeg[0] + t; i < wend[0]; i += kStitchThreads) {
        h[i] = fh[i];
        ok[i] = fv[i];
        if (fv[i] != 0) {
            lg[i] = flg[i];
            se[i] = fse[i];
        }
    }
    int covered = wend[0];
    for (int f = 1; f < windows; ++f) {
        __syncthreads();
        const size_t off = static_cast<size_t>(f) * static_cast<size_t>(bins);
        const double* rlg = flg + off;
        const uint8_t* rv = fv + off;
        const int ob = wbeg[f];
        if (ob >= covered) {  // cannot happen for the engine's windows, which overlap
            if (t == 0) *status = kStitchNoOverlap;
            return;
        }
        const int oe = min(covered, wend[f]);
        // the fallback join: the common valid bin nearest the overlap's midpoint
        const int middle = ob + (oe - ob) / 2;
        double key = INFINITY;
        int bin = 0x7fffffff;
        for (int i = ob + t; i < oe; i += kStitchThreads)
            if (ok[i] != 0 && rv[i] != 0 && finite(lg[i]) && finite(rlg[i])) {
                const double d = static_cast<double>(i > middle ? i - middle : middle - i);
                if (d < key) {
                    key = d;
                    bin = i;
                }
            }
        argmin(key, bin, s_key, s_bin);
        if (bin == 0x7fffffff) {
            if (t == 0) *status = kStitchNoCommonOverlapBin;
            return;
        }
        int join = bin;
        // the slope join, when any slope difference is finite
        key = INFINITY;
        bin = 0x7fffffff;
        for (int i = ob + 2 + t; i + 2 < oe; i += kStitchThreads) {
            if (ok[i] == 0 || rv[i] == 0) continue;
            const double d = fabs(slope_at(lg, ok, i, ob, oe, width) - slope_at(rlg, rv, i, ob, oe, width));
            if (finite(d) && d < key) {
                key = d;
                bin = i;
            }
        }
        argmin(key, bin, s_key, s_bin);
        const bool sloped = bin != 0x7fffffff;
        if (sloped) join = bin;
        const double shift = lg[join] - rlg[join];
        if (t == 0 && joins) {
            wlg_join_quality q{};
            q.join_bin = static_cast<uint64_t>(join);
            double s2 = 0.0, mx = 0.0;
            for (int i = ob; i < oe; ++i)
                if (ok[i] != 0 && rv[i] != 0 && finite(lg[i]) && finite(rlg[i])) {
                    const double d = lg[i] - (rlg[i] + shift);
                    s2 += d * d;
                    mx = fmax(mx, fabs(d));
                    ++q.common_bins;
                }
            q.rmse = q.common_bins ? sqrt(s2 / static_cast<double>(q.common_bins)) : qnan;
            q.max_abs_difference = mx;
            q.slope_difference = sloped ? key : qnan;
            joins[f - 1] = q;
        }
        __syncthreads();  // every read of the left curve in the overlap is done
        for (int i = join + t; i < wend[f]; i += kStitchThreads) {
            h[i] = fh[off + i];
            ok[i] = rv[i];
            if (rv[i] != 0) {
                lg[i] = rlg[i] + shift;
                se[i] = fse[off + i];
            } else {
                lg[i] = qnan;
                se[i] = qnan;
            }
        }
        covered = max(covered, wend[f]);
    }
    __syncthreads();
    if (complete_range) {
        int missing = 0;
        for (int i = t; i < bins; i += kStitchThreads) missing |= ok[i] == 0;
        if (__syncthreads_or(missing)) {
            if (t == 0) *status = kStitchIncomplete;
            return;
        }
        if (t == 0) *status = 0;
        return;  // the host adds N ln 2 - log sum exp (the C library's exp and log)
    }
    // log_sum_exp is finite exactly when some entry is finite; then subtract the peak of the
    // valid bins (std::max(peak, x) keeps peak when x is NaN)
    int any_finite = 0;
    double peak = -INFINITY;
    for (int i = t; i < bins; i += kStitchThreads) {
        any_finite |= finite(lg[i]);
        if (ok[i] != 0 && peak < lg[i]) peak = lg[i];
    }
    if (!__syncthreads_or(any_finite)) {
        if (t == 0) *status = kStitchNoValidBins;
        return;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double p2 = __shfl_down_sync(0xffffffffu, peak, o);
        if (peak < p2) peak = p2;
    }
    if ((t & 31) == 0) s_key[t >> 5] = peak;
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < kStitchThreads / 32; ++w)
            if (s_key[0] < s_key[w]) s_key[0] = s_key[w];
    }
    __syncthreads();
    peak = s_key[0];
    for (int i = t; i < bins; i += kStitchThreads)
        if (ok[i] != 0) lg[i] -= peak;
    if (t == 0) *status = 0;
}

}  // namespace

void launch_stitch(int windows, int bins, const int32_t* wbeg, const int32_t* wend, const double* flg,
                   const uint64_t* fh, const double* fse, const uint8_t* fv, const int* summarize_status,
                   double width, int complete_range, double* lg, uint64_t* h, double* se, uint8_t* ok,
                   wlg_join_quality* joins, int* status, cudaStream_t stream) {
    stitch_kernel<<<1, kStitchThreads, 0, stream>>>(windows, bins, wbeg, wend, flg, fh, fse, fv, summarize_status,
                                                     width, complete_range, lg, h, se, ok, joins, status);
    check_cuda(cudaGetLastError(), "stitch_kernel");
}

}  // namespace wlg
