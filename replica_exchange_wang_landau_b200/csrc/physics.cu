// physics.cu — coupling construction and local fields on the device.
//
//  * dense_build_kernel: DenseCouplings (src/physics.cpp:172-184).  One 32x32 tile of
//    pairs (i < j) per CTA; each pair is evaluated once, in the reference's orientation
//    (displacement r_j - r_i, axes e_i then e_j), and written to both triangles through a
//    shared-memory transpose so both stores are coalesced.
//  * csr_count_kernel / csr_fill_kernel: CsrCouplings (src/physics.cpp:197-223) from a cell
//    grid (cells wider than the cutoff, built on the host at upload): one warp per row visits
//    the sites of its cell and the adjacent ones, evaluates each pair once in the reference's
//    orientation and keeps those within the cutoff, O(N z) instead of the reference's O(N^2)
//    scan.  The row is then sorted by column in shared memory (a bitonic network), which
//    gives the reference's (row, column) order; rows longer than the sort buffer take the
//    scan over all columns in increasing order (csr_scan_fill_kernel).
//  * fields_kernel / energy_kernel: local_fields and total_energy (src/physics.cpp:
//    238-259) with the reference's sequential summation order.
//
// All three are set-up kernels (O(N^2) once per system); the sampling hot path is in
// walker.cu.
#include "engine.hpp"

namespace wlg {

struct SystemView {
    const double* pos;   // n x 3
    const double* axes;  // n x 3
    double box[3];
    int32_t periodic;
    double scale;
    double cutoff;
    int32_t n;
    // the cell grid (CSR only)
    const int32_t* cell_start;  // cells + 1
    const int32_t* cell_sites;  // n, grouped by cell
    const int32_t* site_cell;   // n
    int32_t nc[3];
    int32_t wrap[3];
};

// minimum_image (src/physics.cpp:151-160)
__device__ __forceinline__ void minimum_image(const SystemView& s, double& dx, double& dy, double& dz) {
    if (!s.periodic) return;
    if (s.box[0] > 0.0) dx -= s.box[0] * rint(dx / s.box[0]);
    if (s.box[1] > 0.0) dy -= s.box[1] * rint(dy / s.box[1]);
    if (s.box[2] > 0.0) dz -= s.box[2] * rint(dz / s.box[2]);
}

// pair_for + dipolar_pair (src/physics.cpp:26-30, 162-170) for a < b.  Returns false for
// coincident sites.  `dist` receives norm(d) for the CSR cutoff test.
__device__ __forceinline__ bool pair_value(const SystemView& s, int a, int b, double& value, double& dist) {
    double dx = s.pos[3 * b] - s.pos[3 * a];
    double dy = s.pos[3 * b + 1] - s.pos[3 * a + 1];
    double dz = s.pos[3 * b + 2] - s.pos[3 * a + 2];
    minimum_image(s, dx, dy, dz);
    const double r2 = dx * dx + dy * dy + dz * dz;
    dist = sqrt(r2);
    if (!(r2 > 0.0)) { value = 0.0; return false; }
    const double inv_r = 1.0 / sqrt(r2);
    const double rx = dx * inv_r, ry = dy * inv_r, rz = dz * inv_r;
    const double* ai = s.axes + 3 * a;
    const double* aj = s.axes + 3 * b;
    const double dot_ij = ai[0] * aj[0] + ai[1] * aj[1] + ai[2] * aj[2];
    const double dot_ir = ai[0] * rx + ai[1] * ry + ai[2] * rz;
    const double dot_jr = aj[0] * rx + aj[1] * ry + aj[2] * rz;
    const double angular = dot_ij - 3.0 * dot_ir * dot_jr;
    value = s.scale * angular * inv_r * inv_r * inv_r;
    return true;
}

__global__ void dense_build_kernel(SystemView s, int ld, double* __restrict__ J, int* __restrict__ err) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    __shared__ double tile[32][33];
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bi * 32 + r, j = bj * 32 + threadIdx.x;
        double v = 0.0;
        if (i < s.n && j < s.n && i < j) {
            double dist;
            if (!pair_value(s, i, j, v, dist)) atomicExch(err, 1);
        }
        tile[r][threadIdx.x] = v;
        if (i < ld && j < ld && i <= j) J[static_cast<size_t>(i) * ld + j] = v;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = bj * 32 + r, i = bi * 32 + threadIdx.x;
        if (i < ld && j < ld && i < j) J[static_cast<size_t>(j) * ld + i] = tile[threadIdx.x][r];
    }
}

// Calls f(cell) for the cell of `site` and the cells adjacent to it (at most 27, each once).
template <class F>
__device__ __forceinline__ void for_adjacent_cells(const SystemView& s, int site, F&& f) {
    const int cell = s.site_cell[site];
    const int c0 = cell % s.nc[0], c1 = (cell / s.nc[0]) % s.nc[1], c2 = cell / (s.nc[0] * s.nc[1]);
    const int r0 = s.nc[0] > 1 ? 1 : 0, r1 = s.nc[1] > 1 ? 1 : 0, r2 = s.nc[2] > 1 ? 1 : 0;
    for (int d2 = -r2; d2 <= r2; ++d2) {
        int z = c2 + d2;
        if (s.wrap[2]) z = z < 0 ? z + s.nc[2] : (z >= s.nc[2] ? z - s.nc[2] : z);
        else if (z < 0 || z >= s.nc[2]) continue;
        for (int d1 = -r1; d1 <= r1; ++d1) {
            int y = c1 + d1;
            if (s.wrap[1]) y = y < 0 ? y + s.nc[1] : (y >= s.nc[1] ? y - s.nc[1] : y);
            else if (y < 0 || y >= s.nc[1]) continue;
            for (int d0 = -r0; d0 <= r0; ++d0) {
                int x = c0 + d0;
                if (s.wrap[0]) x = x < 0 ? x + s.nc[0] : (x >= s.nc[0] ? x - s.nc[0] : x);
                else if (x < 0 || x >= s.nc[0]) continue;
                f(x + s.nc[0] * (y + s.nc[1] * z));
            }
        }
    }
}

// One warp per row: count the columns c != row with norm(d) <= cutoff among the sites of the
// adjacent cells.
__global__ void csr_count_kernel(SystemView s, int32_t* __restrict__ counts, int* __restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int row = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (row >= s.n) return;
    int total = 0;
    for_adjacent_cells(s, row, [&](int cell) {
        const int end = s.cell_start[cell + 1];
        for (int q0 = s.cell_start[cell]; q0 < end; q0 += 32) {
            const int q = q0 + lane;
            bool in = false;
            if (q < end) {
                const int c = s.cell_sites[q];
                if (c != row) {
                    double v, dist;
                    const bool ok = pair_value(s, min(row, c), max(row, c), v, dist);
                    in = dist <= s.cutoff;
                    if (in && !ok) atomicExch(err, 1);
                }
            }
            total += __popc(__ballot_sync(0xffffffffu, in));
        }
    });
    if (lane == 0) counts[row] = total;
}

constexpr int kSortCapacity = 1024;  // entries of the per-warp row sort buffer
constexpr int kFillWarps = 4;

// One warp per row: the row's (column, value) pairs from the adjacent cells into shared
// memory, sorted by column with a bitonic network, then stored at ptr[row].  Rows with more
// than kSortCapacity entries are listed in `overflow` for csr_scan_fill_kernel.
__global__ void __launch_bounds__(32 * kFillWarps) csr_fill_kernel(SystemView s, const int32_t* __restrict__ ptr,
                                                                   int32_t* __restrict__ col,
                                                                   double* __restrict__ val64,
                                                                   float* __restrict__ val32,
                                                                   int32_t* __restrict__ overflow,
                                                                   int* __restrict__ overflow_count) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (row >= s.n) return;
    const int count = ptr[row + 1] - ptr[row];
    if (count > kSortCapacity) {
        if (lane == 0) overflow[atomicAdd(overflow_count, 1)] = row;
        return;
    }
    double* vs = reinterpret_cast<double*>(smem) + static_cast<size_t>(warp) * kSortCapacity;
    int32_t* cs = reinterpret_cast<int32_t*>(smem + static_cast<size_t>(kFillWarps) * kSortCapacity * 8) +
                  static_cast<size_t>(warp) * kSortCapacity;
    int at = 0;
    for_adjacent_cells(s, row, [&](int cell) {
        const int end = s.cell_start[cell + 1];
        for (int q0 = s.cell_start[cell]; q0 < end; q0 += 32) {
            const int q = q0 + lane;
            bool in = false;
            int c = 0;
            double v = 0.0;
            if (q < end) {
                c = s.cell_sites[q];
                if (c != row) {
                    double dist;
                    pair_value(s, min(row, c), max(row, c), v, dist);
                    in = dist <= s.cutoff;
                }
            }
            const unsigned mask = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int e = at + __popc(mask & ((1u << lane) - 1u));
                if (e < kSortCapacity) {
                    cs[e] = c;
                    vs[e] = v;
                }
            }
            at += __popc(mask);
        }
    });
    int padded = 1;
    while (padded < count) padded <<= 1;
    for (int e = count + lane; e < padded; e += 32) {
        cs[e] = 0x7fffffff;
        vs[e] = 0.0;
    }
    __syncwarp();
    for (int k = 2; k <= padded; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < padded; i += 32) {
                const int partner = i ^ j;
                if (partner > i) {
                    const bool ascending = (i & k) == 0;
                    const int a = cs[i], b = cs[partner];
                    if ((a > b) == ascending) {
                        cs[i] = b;
                        cs[partner] = a;
                        const double t = vs[i];
                        vs[i] = vs[partner];
                        vs[partner] = t;
                    }
                }
            }
            __syncwarp();
        }
    }
    const int base = ptr[row];
    for (int e = lane; e < count; e += 32) {
        col[base + e] = cs[e];
        val64[base + e] = vs[e];
        if (val32) val32[base + e] = static_cast<float>(vs[e]);
    }
}

// One warp per listed row: all columns in increasing order, compacted with a ballot (the
// reference's order without sorting; O(N) per row).
__global__ void csr_scan_fill_kernel(SystemView s, const int32_t* __restrict__ rows, int count,
                                     const int32_t* __restrict__ ptr, int32_t* __restrict__ col,
                                     double* __restrict__ val64, float* __restrict__ val32) {
    const int lane = threadIdx.x & 31;
    const int k = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (k >= count) return;
    const int row = rows[k];
    int base = ptr[row];
    for (int c0 = 0; c0 < s.n; c0 += 32) {
        const int c = c0 + lane;
        bool in = false;
        double v = 0.0;
        if (c < s.n && c != row) {
            double dist;
            pair_value(s, min(row, c), max(row, c), v, dist);
            in = dist <= s.cutoff;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int at = base + __popc(mask & ((1u << lane) - 1u));
            col[at] = c;
            val64[at] = v;
            if (val32) val32[at] = static_cast<float>(v);
        }
        base += __popc(mask);
    }
}

// Row-scaled BF16 copy: scale_i = max_j |J_ij| (as float), q_ij = bf16(J_ij / scale_i).
__global__ void dense_lowp_kernel(const double* __restrict__ J, int n, int ld, float* __restrict__ J32,
                                  __nv_bfloat16* __restrict__ J16, float* __restrict__ scale) {
    const int row = blockIdx.x;
    __shared__ double red[32];
    double mx = 0.0;
    for (int j = threadIdx.x; j < ld; j += blockDim.x) mx = fmax(mx, fabs(J[static_cast<size_t>(row) * ld + j]));
    for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        mx = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (threadIdx.x == 0) red[0] = mx;
    }
    __syncthreads();
    const float sc = red[0] > 0.0 ? static_cast<float>(red[0]) : 1.0f;
    if (threadIdx.x == 0 && scale) scale[row] = sc;
    for (int j = threadIdx.x; j < ld; j += blockDim.x) {
        const double x = J[static_cast<size_t>(row) * ld + j];
        if (J32) J32[static_cast<size_t>(row) * ld + j] = static_cast<float>(x);
        if (J16) J16[static_cast<size_t>(row) * ld + j] = __double2bfloat16(x / static_cast<double>(sc));
    }
    (void)n;
}

// local_fields for `count` configurations: thread per (config, site), sequential in j.
__global__ void fields_kernel(EngineView v, const int8_t* __restrict__ spins, int64_t spin_stride,
                              double* __restrict__ fields, int64_t field_stride, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= v.n || k >= count) return;
    const int8_t* s = spins + k * spin_stride;
    double sum = 0.0;
    if (!v.csr) {
        for (int j = 0; j < v.n; ++j) sum += v.J64[static_cast<size_t>(j) * v.ld + i] * static_cast<double>(s[j]);
    } else {
        for (int q = v.csr_ptr[i]; q < v.csr_ptr[i + 1]; ++q)
            sum += v.csr_val64[q] * static_cast<double>(s[v.csr_col[q]]);
    }
    fields[k * field_stride + i] = sum;
}

// local_fields of dense couplings for G configurations per block.  Each thread owns one site i
// and keeps G sums; the J column entries J[j][i] are read kFieldPrefetch rows ahead into
// registers, and the configurations' spins are staged as doubles (+-1.0) in shared memory,
// TILE rows at a time, so that a term is one multiply and one add, with one shared-memory
// broadcast (a double2) per two terms.  Every field is still summed sequentially over j with
// the reference's operations (sum += J(i, j) * s_j, no contraction), so the result is the one
// of fields_kernel whatever G is.  A block reads its sites' columns of J once for G
// configurations.  G = 8 is used: G = 32 (64 threads, 128 registers) reads J four times less but
// leaves a quarter of the warps, and the FP64 recompute of 256 walkers at N = 2458 took 0.56 ms
// with it against 0.43 ms with G = 8.
constexpr int kFieldPrefetch = 8;   // rows of J in flight per thread
template <int G, int TILE, int THREADS>
__global__ void __launch_bounds__(THREADS) fields_group_kernel(EngineView v, const int8_t* __restrict__ spins,
                                                                int64_t spin_stride, double* __restrict__ fields,
                                                                int64_t field_stride, int count) {
    __shared__ __align__(16) double sigma[TILE][G];  // row j: the group's spins, contiguous
    const int n = v.n;
    const int k0 = static_cast<int>(blockIdx.y) * G;
    const int group = min(G, count - k0);
    const int i = static_cast<int>(blockIdx.x) * THREADS + static_cast<int>(threadIdx.x);
    const bool site = i < n;
    const double* __restrict__ col = v.J64 + (site ? i : 0);  // J[j][i] at col[j * ld]
    const size_t ld = static_cast<size_t>(v.ld);
    double sum[G];
#pragma unroll
    for (int g = 0; g < G; ++g) sum[g] = 0.0;
    double jv[kFieldPrefetch];
#pragma unroll
    for (int u = 0; u < kFieldPrefetch; ++u) jv[u] = u < n ? col[static_cast<size_t>(u) * ld] : 0.0;
    for (int t0 = 0; t0 < n; t0 += TILE) {
        const int tile = min(TILE, n - t0);
        __syncthreads();  // the previous tile is no longer read
        for (int q = static_cast<int>(threadIdx.x); q < G * TILE; q += THREADS) {
            const int j = q / G, g = q % G;  // consecutive threads: one row, conflict-free stores
            sigma[j][g] = (g < group && j < tile)
                              ? static_cast<double>(spins[static_cast<size_t>(k0 + g) * spin_stride + t0 + j])
                              : 0.0;
        }
        __syncthreads();
        for (int j0 = 0; j0 < tile; j0 += kFieldPrefetch) {
            // the next kFieldPrefetch rows of J, issued before this block of rows is summed
            double jn[kFieldPrefetch];
#pragma unroll
            for (int u = 0; u < kFieldPrefetch; ++u) {
                const int j = t0 + j0 + kFieldPrefetch + u;
                jn[u] = j < n ? col[static_cast<size_t>(j) * ld] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kFieldPrefetch; ++u) {
                if (j0 + u < tile) {
                    const double2* row = reinterpret_cast<const double2*>(&sigma[j0 + u][0]);
#pragma unroll
                    for (int g2 = 0; g2 < G / 2; ++g2) {
                        const double2 sg = row[g2];
                        sum[2 * g2] += jv[u] * sg.x;
                        sum[2 * g2 + 1] += jv[u] * sg.y;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kFieldPrefetch; ++u) jv[u] = jn[u];
        }
    }
    if (!site) return;
#pragma unroll
    for (int g = 0; g < G; ++g)
        if (g < group) fields[static_cast<size_t>(k0 + g) * field_stride + i] = sum[g];
}

// total_energy (src/physics.cpp:253-259): E = sum over i of 0.5 * s_i * h_i, in site order.  One
// warp per configuration: the lanes form 32 terms at a time (coalesced loads, the next chunk's
// issued before this chunk is added) and every lane adds them in order from shared memory, so
// the sum is the reference's sequential one.
constexpr int kEnergyWarps = 4;
__global__ void __launch_bounds__(32 * kEnergyWarps) energy_kernel(int n, const int8_t* __restrict__ spins,
                                                                   int64_t spin_stride,
                                                                   const double* __restrict__ fields,
                                                                   int64_t field_stride, double* __restrict__ out,
                                                                   int count) {
    __shared__ double terms[kEnergyWarps][32];
    const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
    const int k = static_cast<int>(blockIdx.x) * kEnergyWarps + warp;
    if (k >= count) return;  // whole warps only: the kernel has no block-wide barrier
    const int8_t* s = spins + static_cast<size_t>(k) * spin_stride;
    const double* f = fields + static_cast<size_t>(k) * field_stride;
    int8_t sn = lane < n ? s[lane] : 0;
    double fn = lane < n ? f[lane] : 0.0;
    double e = 0.0;
    for (int base = 0; base < n; base += 32) {
        terms[warp][lane] = 0.5 * static_cast<double>(sn) * fn;
        __syncwarp();
        const int next = base + 32 + lane;  // the next chunk's loads, in flight during the adds
        sn = next < n ? s[next] : 0;
        fn = next < n ? f[next] : 0.0;
        const int m = min(32, n - base);
        for (int q = 0; q < m; ++q) e += terms[warp][q];
        __syncwarp();
    }
    if (lane == 0) out[k] = e;
}

// ---- host launchers ------------------------------------------------------------------

static SystemView make_view(const DeviceSystem& d) {
    SystemView s{};
    s.pos = d.pos.get<double>();
    s.axes = d.axes.get<double>();
    for (int k = 0; k < 3; ++k) s.box[k] = d.box[k];
    s.periodic = d.periodic;
    s.scale = d.scale;
    s.cutoff = d.cutoff;
    s.n = static_cast<int32_t>(d.n);
    s.cell_start = d.cell_start.get<int32_t>();
    s.cell_sites = d.cell_sites.get<int32_t>();
    s.site_cell = d.site_cell.get<int32_t>();
    for (int k = 0; k < 3; ++k) {
        s.nc[k] = d.cells[k];
        s.wrap[k] = d.cell_wrap[k];
    }
    return s;
}

void launch_dense_build(const double* pos, const double* axes, const double* box, int periodic, double scale, int n,
                        int ld, double* J, int* err, cudaStream_t stream) {
    SystemView s{};
    s.pos = pos;
    s.axes = axes;
    for (int k = 0; k < 3; ++k) s.box[k] = box[k];
    s.periodic = periodic;
    s.scale = scale;
    s.cutoff = 0.0;
    s.n = n;
    const int tiles = (ld + 31) / 32;
    dense_build_kernel<<<dim3(tiles, tiles), dim3(32, 8), 0, stream>>>(s, ld, J, err);
    check_cuda(cudaGetLastError(), "dense_build_kernel");
}

// The FP32 / BF16 (+ row scale) copies of a dense FP64 J.
static void build_dense_lowp(DeviceSystem& d, int precision, cudaStream_t stream) {
    if (precision == WLG_PRECISION_FP32) d.J32.allocate(d.ld * d.ld * sizeof(float));
    if (precision == WLG_PRECISION_BF16) {
        d.J16.allocate(d.ld * d.ld * sizeof(__nv_bfloat16));
        d.Jscale.allocate(d.ld * sizeof(float));
    }
    if (precision != WLG_PRECISION_FP64) {
        dense_lowp_kernel<<<static_cast<unsigned>(d.ld), 256, 0, stream>>>(
            d.J64.get<double>(), static_cast<int>(d.n), static_cast<int>(d.ld), d.J32.get<float>(),
            d.J16.get<__nv_bfloat16>(), d.Jscale.get<float>());
        check_cuda(cudaGetLastError(), "dense_lowp_kernel");
    }
}

// The ELLPACK copy read by the CSR sweep (rows of at most 256 couplings; zmax = longest row).
static void build_ellpack(DeviceSystem& d, int precision, int32_t zmax, cudaStream_t stream) {
    const int n = static_cast<int>(d.n);
    int32_t width = 32;
    while (width < zmax && width < 256) width *= 2;
    if (zmax <= 256) {
        const size_t entries = static_cast<size_t>(n) * static_cast<size_t>(width);
        d.ell_col.allocate(entries * sizeof(int32_t));
        if (precision == WLG_PRECISION_FP32) d.ell_val32.allocate(entries * sizeof(float));
        else d.ell_val64.allocate(entries * sizeof(double));
        launch_ell_fill(n, width, d.csr_ptr.get<int32_t>(), d.csr_col.get<int32_t>(), d.csr_val64.get<double>(),
                        d.csr_val32.get<float>(), d.ell_col.get<int32_t>(), d.ell_val64.get<double>(),
                        d.ell_val32.get<float>(), stream);
        d.ell_width = width;
    }
}

void upload_couplings(const wlg_couplings& j, DeviceSystem& d, int precision, cudaStream_t stream) {
    d.n = j.n;
    d.ld = (j.n + 15) / 16 * 16;
    d.csr = j.dense == nullptr;
    const uint64_t n = j.n;
    if (!d.csr) {
        d.J64.allocate(d.ld * d.ld * sizeof(double));
        check_cuda(cudaMemsetAsync(d.J64.ptr, 0, d.J64.bytes, stream), "memset J");
        check_cuda(cudaMemcpy2DAsync(d.J64.ptr, d.ld * sizeof(double), j.dense, n * sizeof(double), n * sizeof(double),
                                     n, cudaMemcpyHostToDevice, stream),
                   "copy J");
        build_dense_lowp(d, precision, stream);
        check_cuda(cudaStreamSynchronize(stream), "sync");
        return;
    }
    const size_t nnz = static_cast<size_t>(j.nnz);
    std::vector<int32_t> ptr(n + 1), col(std::max<size_t>(1, nnz));
    std::vector<float> v32;
    int32_t zmax = 0;
    for (uint64_t r = 0; r <= n; ++r) ptr[r] = static_cast<int32_t>(j.row_offsets[r]);
    for (uint64_t r = 0; r < n; ++r) zmax = std::max(zmax, ptr[r + 1] - ptr[r]);
    for (size_t k = 0; k < nnz; ++k) col[k] = static_cast<int32_t>(j.columns[k]);
    d.nnz = nnz;
    d.csr_ptr.allocate(ptr.size() * sizeof(int32_t));
    d.csr_col.allocate(col.size() * sizeof(int32_t));
    d.csr_val64.allocate(std::max<size_t>(1, nnz) * sizeof(double));
    check_cuda(cudaMemcpyAsync(d.csr_ptr.ptr, ptr.data(), d.csr_ptr.bytes, cudaMemcpyHostToDevice, stream), "copy ptr");
    check_cuda(cudaMemcpyAsync(d.csr_col.ptr, col.data(), nnz * sizeof(int32_t), cudaMemcpyHostToDevice, stream),
               "copy columns");
    check_cuda(cudaMemcpyAsync(d.csr_val64.ptr, j.values, nnz * sizeof(double), cudaMemcpyHostToDevice, stream),
               "copy values");
    if (precision == WLG_PRECISION_FP32) {
        v32.resize(std::max<size_t>(1, nnz));
        for (size_t k = 0; k < nnz; ++k) v32[k] = static_cast<float>(j.values[k]);  // as csr_fill_kernel rounds
        d.csr_val32.allocate(v32.size() * sizeof(float));
        check_cuda(cudaMemcpyAsync(d.csr_val32.ptr, v32.data(), nnz * sizeof(float), cudaMemcpyHostToDevice, stream),
                   "copy values");
    }
    build_ellpack(d, precision, zmax, stream);
    check_cuda(cudaStreamSynchronize(stream), "sync");
}

void build_couplings(DeviceSystem& d, int precision, cudaStream_t stream) {
    const SystemView s = make_view(d);
    DeviceBuffer err(sizeof(int));
    check_cuda(cudaMemsetAsync(err.ptr, 0, sizeof(int), stream), "memset");
    const int n = static_cast<int>(d.n);
    if (!d.csr) {
        d.J64.allocate(d.ld * d.ld * sizeof(double));
        check_cuda(cudaMemsetAsync(d.J64.ptr, 0, d.J64.bytes, stream), "memset J");
        const int tiles = static_cast<int>((d.ld + 31) / 32);
        dense_build_kernel<<<dim3(tiles, tiles), dim3(32, 8), 0, stream>>>(s, static_cast<int>(d.ld),
                                                                           d.J64.get<double>(), err.get<int>());
        check_cuda(cudaGetLastError(), "dense_build_kernel");
        build_dense_lowp(d, precision, stream);
    } else {
        DeviceBuffer counts(static_cast<size_t>(n) * sizeof(int32_t));
        const int warps_per_block = 8;
        const unsigned blocks = static_cast<unsigned>((n + warps_per_block - 1) / warps_per_block);
        csr_count_kernel<<<blocks, 32 * warps_per_block, 0, stream>>>(s, counts.get<int32_t>(), err.get<int>());
        check_cuda(cudaGetLastError(), "csr_count_kernel");
        std::vector<int32_t> host_counts(static_cast<size_t>(n));
        check_cuda(cudaMemcpyAsync(host_counts.data(), counts.ptr, counts.bytes, cudaMemcpyDeviceToHost, stream),
                   "copy counts");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        std::vector<int32_t> ptr(static_cast<size_t>(n) + 1, 0);
        int64_t total = 0;
        for (int i = 0; i < n; ++i) {
            total += host_counts[static_cast<size_t>(i)];
            if (total > INT32_MAX) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR has more than 2^31 couplings");
            ptr[static_cast<size_t>(i) + 1] = static_cast<int32_t>(total);
        }
        d.nnz = static_cast<uint64_t>(total);
        d.csr_ptr.allocate(ptr.size() * sizeof(int32_t));
        check_cuda(cudaMemcpyAsync(d.csr_ptr.ptr, ptr.data(), d.csr_ptr.bytes, cudaMemcpyHostToDevice, stream),
                   "copy ptr");
        const size_t nnz = std::max<size_t>(1, static_cast<size_t>(total));
        d.csr_col.allocate(nnz * sizeof(int32_t));
        d.csr_val64.allocate(nnz * sizeof(double));
        if (precision == WLG_PRECISION_FP32) d.csr_val32.allocate(nnz * sizeof(float));
        DeviceBuffer overflow(static_cast<size_t>(n) * sizeof(int32_t) + sizeof(int));
        int* overflow_count = reinterpret_cast<int*>(overflow.get<unsigned char>() + static_cast<size_t>(n) * 4);
        check_cuda(cudaMemsetAsync(overflow_count, 0, sizeof(int), stream), "memset");
        const size_t fill_smem = static_cast<size_t>(kFillWarps) * kSortCapacity * (8 + 4);
        csr_fill_kernel<<<static_cast<unsigned>((n + kFillWarps - 1) / kFillWarps), 32 * kFillWarps, fill_smem, stream>>>(
            s, d.csr_ptr.get<int32_t>(), d.csr_col.get<int32_t>(), d.csr_val64.get<double>(), d.csr_val32.get<float>(),
            overflow.get<int32_t>(), overflow_count);
        check_cuda(cudaGetLastError(), "csr_fill_kernel");
        int long_rows = 0;
        check_cuda(cudaMemcpyAsync(&long_rows, overflow_count, sizeof(int), cudaMemcpyDeviceToHost, stream), "copy");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        if (long_rows > 0) {
            csr_scan_fill_kernel<<<static_cast<unsigned>((long_rows + warps_per_block - 1) / warps_per_block),
                                   32 * warps_per_block, 0, stream>>>(s, overflow.get<int32_t>(), long_rows,
                                                                      d.csr_ptr.get<int32_t>(), d.csr_col.get<int32_t>(),
                                                                      d.csr_val64.get<double>(), d.csr_val32.get<float>());
            check_cuda(cudaGetLastError(), "csr_scan_fill_kernel");
        }
        int32_t zmax = 0;
        for (int32_t c : host_counts) zmax = std::max(zmax, c);
        build_ellpack(d, precision, zmax, stream);
    }
    int host_err = 0;
    check_cuda(cudaMemcpyAsync(&host_err, err.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream), "copy err");
    check_cuda(cudaStreamSynchronize(stream), "sync");
    if (host_err) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Coincident dipole sites");
}

void compute_fields(const EngineView& v, const int8_t* spins, int64_t spin_stride, double* fields,
                    int64_t field_stride, double* energies, int count, cudaStream_t stream) {
    if (count <= 0) return;
    if (!v.csr && count > 1) {
        constexpr int G = 8, TILE = 256, THREADS = 128;
        const dim3 grid(static_cast<unsigned>((v.n + THREADS - 1) / THREADS), static_cast<unsigned>((count + G - 1) / G));
        fields_group_kernel<G, TILE, THREADS><<<grid, THREADS, 0, stream>>>(v, spins, spin_stride, fields, field_stride,
                                                                             count);
        check_cuda(cudaGetLastError(), "fields_group_kernel");
    } else {
        const dim3 grid(static_cast<unsigned>((v.n + 127) / 128), static_cast<unsigned>(count));
        fields_kernel<<<grid, 128, 0, stream>>>(v, spins, spin_stride, fields, field_stride, count);
        check_cuda(cudaGetLastError(), "fields_kernel");
    }
    if (energies) {
        energy_kernel<<<static_cast<unsigned>((count + kEnergyWarps - 1) / kEnergyWarps), 32 * kEnergyWarps, 0, stream>>>(
            v.n, spins, spin_stride, fields, field_stride, energies, count);
        check_cuda(cudaGetLastError(), "energy_kernel");
    }
}

}  // namespace wlg
