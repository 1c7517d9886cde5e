// precision.cu — the periodic FP64 recompute of a mixed-precision run (no counterpart in
// the reference, which stores J in FP64 only).
//
// With J stored in FP32, or BF16 with a per-row scale, every accepted flip adds
// m * J_lowp[i][j] to the FP64 local fields, so the fields and the walker energy drift from
// their exact values.  Every recompute interval the engine rebuilds all configurations'
// fields and energies from the resident FP64 J with the reference's own summation order
// (local_fields / total_energy, src/physics.cpp:238-259; fields_kernel / energy_kernel),
// and resync_kernel then, per walker:
//   * measures the drift: max_j |h_j - h64_j| and |E - E64|;
//   * replaces the fields and the energy by the FP64 values and re-derives the current bin
//     from E64 (bin index and energy stay FP64), unless E64 falls outside the walker's
//     window: that resync is deferred to the next interval and counted, so a walker is never
//     moved out of its window by a correction.
// The drift maxima, recompute, deferral and bin-change counts accumulate in a
// PrecisionReport on the device, read by wlg_engine_precision_report.  A recompute after the
// epoch that terminated the run changes nothing and is not counted.
#include "engine.hpp"
#include "walker_dev.cuh"

namespace wlg {

namespace {

__device__ __forceinline__ double warp_max_double(double x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(kFull, x, o));
    return x;
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* at, double x) {
    atomicMax(at, static_cast<unsigned long long>(__double_as_longlong(x)));
}

__global__ void resync_kernel(EngineView v, const double* __restrict__ rfields, const double* __restrict__ renergy,
                              PrecisionReport* report) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    // a run that has terminated is not corrected any more (its results are final)
    if (w >= v.walkers || v.ctl->error != 0 || v.ctl->done != 0) return;
    if (w == 0 && lane == 0) atomicAdd(&report->recomputes, 1ULL);
    WalkerState& st = v.ws[w];
    const size_t base = static_cast<size_t>(st.slot) * static_cast<size_t>(v.ld);
    double* f = v.fields + base;
    const double* rf = rfields + base;
    double dmax = 0.0;
    for (int j = lane; j < v.n; j += 32) dmax = fmax(dmax, fabs(f[j] - rf[j]));
    dmax = warp_max_double(dmax);
    const double e64 = renergy[st.slot];
    const double de = fabs(st.energy - e64);
    const int64_t bin = grid_index(v.grid, e64);
    const bool ok = bin >= v.win_begin[st.window] && bin < v.win_end[st.window];
    if (ok)
        for (int j = lane; j < v.n; j += 32) f[j] = rf[j];
    __syncwarp();
    if (lane == 0) {
        atomic_max_nonneg(&report->max_field_drift_bits, dmax);
        atomic_max_nonneg(&report->max_energy_drift_bits, de);
        if (ok) {
            if (bin != st.cur_bin) {
                st.cur_bin = static_cast<int32_t>(bin);
                atomicAdd(&report->bin_changes, 1ULL);
            }
            st.energy = e64;
            atomicAdd(&report->resynced, 1ULL);
        } else {
            atomicAdd(&report->deferred, 1ULL);
        }
    }
}

}  // namespace

void launch_resync(const EngineView& v, const double* rfields, const double* renergy, PrecisionReport* report,
                   cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((static_cast<size_t>(v.walkers) * 32 + 255) / 256);
    resync_kernel<<<blocks, 256, 0, stream>>>(v, rfields, renergy, report);
    check_cuda(cudaGetLastError(), "resync_kernel");
}

}  // namespace wlg
