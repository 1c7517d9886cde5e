// noalloc.cu — local fields and energies without any device allocation.
//
// wlg_local_fields builds the coupling matrix and stages spins, fields and energies in
// device buffers it allocates (from the device's memory pool).  Some callers cannot allow
// that: a host that has already handed nearly all device memory to its own pool (a caching
// allocator reserves it up front), code that must not add the synchronisation a device
// allocation can cause, or a plugin host that forbids allocation once it has started.  For them this
// file keeps every intermediate in one statically sized device array instead.
//
// The array is a file-scope __device__ object, so every GPU that loads the library holds
// it until the process exits (kScratchBytes, 18 MiB).  Host code may not use its name as a
// device address; every call looks the device address up with cudaGetSymbolAddress, with
// the calling thread's device current (cheap, and it allocates nothing).  Looking it up on
// every call rather than caching it keeps the address valid after the host resets the
// device (cudaDeviceReset reloads the module at a new address).  The first call on a device
// loads the library's device code and should come before any stream capture.  All calls
// share the array and it keeps the last call's contents: the regions that must start at
// zero (the coupling matrix with its padding, the error flag) are cleared on every call,
// and calls that overlap on the GPU (from several host threads at once) race on the array.
// Work is issued on the legacy default stream, which synchronises with blocking streams, so
// no call may run while another thread holds a global-mode stream capture.

#include "engine.hpp"

namespace wlg {

namespace {

constexpr int kMaxSpins = 1024;                                   // dense systems up to 1024 sites
constexpr size_t kJBytes = size_t{kMaxSpins} * kMaxSpins * 8;     // 8 MiB coupling matrix
constexpr size_t kGeomBytes = size_t{kMaxSpins} * 3 * 8;          // positions, then axes
constexpr size_t kMaxValues = size_t{1} << 20;                    // count x n spins / fields
constexpr size_t kMaxConfigs = size_t{1} << 16;                   // count
constexpr size_t kOffJ = 0;
constexpr size_t kOffPos = kOffJ + kJBytes;
constexpr size_t kOffAxes = kOffPos + kGeomBytes;
constexpr size_t kOffErr = kOffAxes + kGeomBytes;
constexpr size_t kOffSpins = kOffErr + 256;
constexpr size_t kOffFields = kOffSpins + kMaxValues;
constexpr size_t kOffEnergies = kOffFields + kMaxValues * 8;
constexpr size_t kScratchBytes = kOffEnergies + kMaxConfigs * 8;  // 18,022,656 bytes

}  // namespace

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// The device address of g_noalloc_scratch on the current device, looked up on every call.
unsigned char* scratch_on_current_device() {
    void* p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    if (!p) throw WlgError(WLG_ERR_DEVICE, "cudaGetSymbolAddress returned a null address");
    return static_cast<unsigned char*>(p);
}

}  // namespace

void local_fields_noalloc(const wlg_system& s, const int8_t* spins, uint64_t count, double* fields,
                          double* energies) {
    validate_system(s);
    if (s.cutoff > 0.0)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT,
                       "wlg_local_fields_noalloc supports dense couplings only (cutoff must be 0)");
    const uint64_t n = s.n;
    const uint64_t ld = (n + 15) / 16 * 16;
    if (ld > static_cast<uint64_t>(kMaxSpins))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "wlg_local_fields_noalloc supports at most " +
                                                     std::to_string(kMaxSpins) + " sites; got " + std::to_string(n));
    if (count > kMaxConfigs || count * n > kMaxValues)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT,
                       "wlg_local_fields_noalloc takes at most " + std::to_string(kMaxConfigs) +
                           " configurations and " + std::to_string(kMaxValues) + " spins per call; got " +
                           std::to_string(count) + " x " + std::to_string(n));
    for (uint64_t k = 0; k < count * n; ++k)
        if (spins[k] != 1 && spins[k] != -1) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Spins must be +/-1");
    if (count == 0) return;
    unsigned char* base = scratch_on_current_device();
    double* J = reinterpret_cast<double*>(base + kOffJ);
    double* pos = reinterpret_cast<double*>(base + kOffPos);
    double* axes = reinterpret_cast<double*>(base + kOffAxes);
    int* err = reinterpret_cast<int*>(base + kOffErr);
    int8_t* d_spins = reinterpret_cast<int8_t*>(base + kOffSpins);
    double* d_fields = reinterpret_cast<double*>(base + kOffFields);
    double* d_energies = reinterpret_cast<double*>(base + kOffEnergies);
    cudaStream_t stream = nullptr;  // legacy default stream

    check_cuda(cudaMemsetAsync(J, 0, ld * ld * 8, stream), "memset J");
    check_cuda(cudaMemsetAsync(err, 0, sizeof(int), stream), "memset flag");
    check_cuda(cudaMemcpyAsync(pos, s.positions, n * 3 * 8, cudaMemcpyHostToDevice, stream), "copy positions");
    check_cuda(cudaMemcpyAsync(axes, s.axes, n * 3 * 8, cudaMemcpyHostToDevice, stream), "copy axes");
    launch_dense_build(pos, axes, s.box, s.periodic != 0, s.coupling_scale, static_cast<int>(n), static_cast<int>(ld), J,
                       err, stream);
    check_cuda(cudaMemcpyAsync(d_spins, spins, count * n, cudaMemcpyHostToDevice, stream), "copy spins");
    EngineView v{};
    v.n = static_cast<int32_t>(n);
    v.ld = static_cast<int32_t>(ld);
    v.csr = 0;
    v.J64 = J;
    compute_fields(v, d_spins, static_cast<int64_t>(n), d_fields, static_cast<int64_t>(n), d_energies,
                   static_cast<int>(count), stream);
    int host_err = 0;
    check_cuda(cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, stream), "copy flag");
    check_cuda(cudaMemcpyAsync(fields, d_fields, count * n * 8, cudaMemcpyDeviceToHost, stream), "copy fields");
    if (energies)
        check_cuda(cudaMemcpyAsync(energies, d_energies, count * 8, cudaMemcpyDeviceToHost, stream), "copy energies");
    check_cuda(cudaStreamSynchronize(stream), "local_fields_noalloc");
    if (host_err) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Coincident dipole sites");
}

}  // namespace wlg
