// host.cpp — host-side pieces that need no GPU: validation with the reference's messages,
// the energy grid, the window partition, geometry upload and the WLCHKP checkpoint format.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <vector>

#include "engine.hpp"

namespace wlg {

namespace {
double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
}  // namespace

// Geometry::validate (src/physics.cpp:34-56)
void validate_system(const wlg_system& s) {
    if (s.n == 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Geometry contains no sites");
    if (!s.positions || !s.axes) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Geometry positions/axes size mismatch");
    if (s.periodic) {
        for (int k = 0; k < 3; ++k)
            if (!(std::isfinite(s.box[k]) && s.box[k] >= 0.0))
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Periodic box lengths must be finite and non-negative");
        if (s.box[0] == 0.0 && s.box[1] == 0.0 && s.box[2] == 0.0)
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "At least one periodic box length must be positive");
    }
    for (uint64_t i = 0; i < s.n; ++i) {
        const double* p = s.positions + 3 * i;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]))
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Site coordinates must be finite");
        const double length = std::sqrt(dot3(s.axes + 3 * i, s.axes + 3 * i));
        if (std::abs(length - 1.0) > 1e-10) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Ising axes must be normalized");
    }
    if (s.n > static_cast<uint64_t>(std::numeric_limits<int32_t>::max() / 2))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Too many sites for one device system");
}

// Prebuilt couplings must be what the reference's backends produce: a symmetric matrix with
// a zero diagonal and finite values (DenseCouplings fills both triangles with the same pair
// value, src/physics.cpp:172-188; CsrCouplings stores every pair in both directions, sorted
// by (row, column), src/physics.cpp:197-223).  The engine's sweeps read a row of J as the
// column add_flip_delta reads, which is only the same thing for a symmetric J.
void validate_couplings(const wlg_couplings& j) {
    const uint64_t n = j.n;
    if (n == 0) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings contain no sites");
    if (n > static_cast<uint64_t>(std::numeric_limits<int32_t>::max() / 2))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Too many sites for one device system");
    if (j.dense) {
        for (uint64_t r = 0; r < n; ++r) {
            if (j.dense[r * n + r] != 0.0)
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must have a zero diagonal");
            for (uint64_t c = r + 1; c < n; ++c) {
                const double a = j.dense[r * n + c], b = j.dense[c * n + r];
                if (!std::isfinite(a)) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must be finite");
                if (std::memcmp(&a, &b, sizeof a) != 0)
                    throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must be symmetric");
            }
        }
        return;
    }
    if (!j.row_offsets || (j.nnz > 0 && (!j.columns || !j.values)))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR couplings need row offsets, columns and values");
    if (j.row_offsets[0] != 0 || j.row_offsets[n] != j.nnz)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR row offsets must start at 0 and end at nnz");
    if (j.nnz > static_cast<uint64_t>(std::numeric_limits<int32_t>::max()))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR has more than 2^31 couplings");
    for (uint64_t r = 0; r < n; ++r) {
        const uint64_t b = j.row_offsets[r], e = j.row_offsets[r + 1];
        if (e < b || e > j.nnz) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR row offsets must be non-decreasing");
        for (uint64_t k = b; k < e; ++k) {
            const uint64_t c = j.columns[k];
            if (c >= n) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR column out of range");
            if (c == r) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must have a zero diagonal");
            if (k > b && c <= j.columns[k - 1])
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "CSR columns must ascend within a row");
            if (!std::isfinite(j.values[k])) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must be finite");
        }
    }
    for (uint64_t r = 0; r < n; ++r)
        for (uint64_t k = j.row_offsets[r]; k < j.row_offsets[r + 1]; ++k) {
            const uint64_t c = j.columns[k];
            const uint64_t* first = j.columns + j.row_offsets[c];
            const uint64_t* last = j.columns + j.row_offsets[c + 1];
            const uint64_t* at = std::lower_bound(first, last, r);
            if (at == last || *at != r ||
                std::memcmp(&j.values[at - j.columns], &j.values[k], sizeof(double)) != 0)
                throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Couplings must be symmetric");
        }
}

// EnergyGrid::validate (src/wang_landau.cpp:13-20)
void validate_grid(double mn, double mx, double w) {
    if (!std::isfinite(mn) || !std::isfinite(mx) || !std::isfinite(w) || !(mx > mn) || !(w > 0.0))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid energy grid");
    const double count = (mx - mn) / w;
    if (std::abs(count - std::round(count)) > 1e-9 * std::max(1.0, count))
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Energy range must be an integer multiple of bin width");
}

// EnergyGrid::bins (src/wang_landau.cpp:22-25)
uint64_t grid_bins(double mn, double mx, double w) {
    validate_grid(mn, mx, w);
    return static_cast<uint64_t>(std::llround((mx - mn) / w));
}

// partition_windows (src/wang_landau.cpp:40-61)
std::vector<uint64_t> partition_windows(uint64_t bins, uint64_t count, double overlap) {
    if (bins == 0 || count == 0 || count > bins || overlap < 0.0 || overlap >= 1.0)
        throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Invalid energy-window partition");
    if (count == 1) return {0, bins};
    const double denominator = 1.0 + static_cast<double>(count - 1) * (1.0 - overlap);
    auto size = static_cast<uint64_t>(std::ceil(static_cast<double>(bins) / denominator));
    size = std::max<uint64_t>(2, std::min(size, bins));
    const uint64_t span = bins - size;
    std::vector<uint64_t> out(2 * count);
    for (uint64_t w = 0; w < count; ++w) {
        const auto begin = static_cast<uint64_t>(
            std::llround(static_cast<double>(w * span) / static_cast<double>(count - 1)));
        out[2 * w] = begin;
        out[2 * w + 1] = begin + size;
    }
    out[2 * count - 1] = bins;
    for (uint64_t w = 1; w < count; ++w)
        if (out[2 * w] >= out[2 * (w - 1) + 1])
            throw WlgError(WLG_ERR_INVALID_ARGUMENT, "Energy windows do not overlap; increase overlap or bins");
    return out;
}

void upload_system(const wlg_system& s, DeviceSystem& d, cudaStream_t stream) {
    d.n = s.n;
    d.ld = (s.n + 15) / 16 * 16;
    for (int k = 0; k < 3; ++k) d.box[k] = s.box[k];
    d.periodic = s.periodic != 0;
    d.scale = s.coupling_scale;
    d.cutoff = s.cutoff;
    d.csr = s.cutoff > 0.0;
    d.pos.allocate(s.n * 3 * sizeof(double));
    d.axes.allocate(s.n * 3 * sizeof(double));
    check_cuda(cudaMemcpyAsync(d.pos.ptr, s.positions, s.n * 3 * sizeof(double), cudaMemcpyHostToDevice, stream),
               "copy positions");
    check_cuda(cudaMemcpyAsync(d.axes.ptr, s.axes, s.n * 3 * sizeof(double), cudaMemcpyHostToDevice, stream),
               "copy axes");
    if (d.csr) upload_cell_grid(s, d, stream);
}

// The cell grid of the CSR build.  Along a periodic axis (box length L > 0) the cells divide
// [0, L) into nc = floor(L / w) equal cells, w = cutoff * (1 + 1e-6), and a position is
// wrapped into [0, L) first; along an open axis they are w wide from the smallest
// coordinate.  Every cell is then wider than the cutoff, so two sites whose minimum-image
// distance is within the cutoff lie in the same or adjacent cells (adjacency wrapping
// around periodic axes); the slack of 1e-6 covers rounding in the cell assignment.  A
// periodic axis with fewer than three cells becomes a single cell, since its neighbours on
// both sides would coincide.  The grid is coarsened (never below the cutoff width) when it
// would have more than 8n + 64 cells.  Sites are listed per cell in increasing index.
void upload_cell_grid(const wlg_system& s, DeviceSystem& d, cudaStream_t stream) {
    const uint64_t n = s.n;
    const double w = s.cutoff * (1.0 + 1e-6);
    int64_t nc[3];
    double lo[3], extent[3], width[3];
    bool wrap[3];
    for (int k = 0; k < 3; ++k) {
        wrap[k] = s.periodic != 0 && s.box[k] > 0.0;
        double mn = std::numeric_limits<double>::infinity(), mx = -mn;
        for (uint64_t i = 0; i < n; ++i) {
            mn = std::min(mn, s.positions[3 * i + k]);
            mx = std::max(mx, s.positions[3 * i + k]);
        }
        lo[k] = mn;
        extent[k] = mx - mn;
        if (wrap[k]) {
            const double cells = std::min(std::floor(s.box[k] / w), 4096.0);
            nc[k] = cells >= 3.0 ? static_cast<int64_t>(cells) : 1;
            width[k] = s.box[k] / static_cast<double>(nc[k]);
        } else {
            width[k] = extent[k] / w > 4095.0 ? extent[k] / 4095.0 : w;
            nc[k] = static_cast<int64_t>(std::floor(extent[k] / width[k])) + 1;
        }
    }
    const auto total = [&]() { return nc[0] * nc[1] * nc[2]; };
    while (total() > static_cast<int64_t>(8 * n + 64)) {
        int k = 0;
        for (int q = 1; q < 3; ++q)
            if (nc[q] > nc[k]) k = q;
        if (wrap[k]) {
            nc[k] = nc[k] / 2 >= 3 ? nc[k] / 2 : 1;
            width[k] = s.box[k] / static_cast<double>(nc[k]);
        } else {
            width[k] *= 2.0;
            nc[k] = static_cast<int64_t>(std::floor(extent[k] / width[k])) + 1;
        }
    }
    std::vector<int32_t> cell_of(n), count(static_cast<size_t>(total()) + 1, 0);
    for (uint64_t i = 0; i < n; ++i) {
        int64_t c[3];
        for (int k = 0; k < 3; ++k) {
            const double x = s.positions[3 * i + k];
            double u;
            if (wrap[k]) {
                u = x / s.box[k];
                u = (u - std::floor(u)) * static_cast<double>(nc[k]);
            } else {
                u = (x - lo[k]) / width[k];
            }
            c[k] = std::min<int64_t>(nc[k] - 1, std::max<int64_t>(0, static_cast<int64_t>(u)));
        }
        cell_of[i] = static_cast<int32_t>(c[0] + nc[0] * (c[1] + nc[1] * c[2]));
        ++count[static_cast<size_t>(cell_of[i]) + 1];
    }
    for (size_t c = 1; c < count.size(); ++c) count[c] += count[c - 1];
    std::vector<int32_t> sites(n), fill(count.begin(), count.end() - 1);
    for (uint64_t i = 0; i < n; ++i) sites[static_cast<size_t>(fill[static_cast<size_t>(cell_of[i])]++)] = static_cast<int32_t>(i);
    for (int k = 0; k < 3; ++k) {
        d.cells[k] = static_cast<int32_t>(nc[k]);
        d.cell_wrap[k] = wrap[k] ? 1 : 0;
    }
    d.cell_start.allocate(count.size() * sizeof(int32_t));
    d.cell_sites.allocate(n * sizeof(int32_t));
    d.site_cell.allocate(n * sizeof(int32_t));
    check_cuda(cudaMemcpyAsync(d.cell_start.ptr, count.data(), d.cell_start.bytes, cudaMemcpyHostToDevice, stream),
               "copy cells");
    check_cuda(cudaMemcpyAsync(d.cell_sites.ptr, sites.data(), d.cell_sites.bytes, cudaMemcpyHostToDevice, stream),
               "copy cells");
    check_cuda(cudaMemcpyAsync(d.site_cell.ptr, cell_of.data(), d.site_cell.bytes, cudaMemcpyHostToDevice, stream),
               "copy cells");
    check_cuda(cudaStreamSynchronize(stream), "sync");  // the host vectors go out of scope
}

// ---- checkpoint (src/io.cpp:539-572) ---------------------------------------------------

namespace {
template <class T> void put(std::ofstream& out, const T& v) { out.write(reinterpret_cast<const char*>(&v), sizeof v); }
template <class T> void put_vec(std::ofstream& out, const T* data, uint64_t count) {
    put(out, count);
    out.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(count * sizeof(T)));
}
template <class T> bool get(std::ifstream& in, T& v) {
    in.read(reinterpret_cast<char*>(&v), sizeof v);
    return static_cast<bool>(in);
}
template <class T> bool get_vec(std::ifstream& in, std::vector<T>& v, std::string& error) {
    uint64_t size = 0;
    if (!get(in, size)) { error = "Truncated checkpoint"; return false; }
    if (size > 1'000'000'000ULL) { error = "Unreasonable checkpoint vector size"; return false; }
    v.resize(static_cast<size_t>(size));
    in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(size * sizeof(T)));
    if (!in) { error = "Truncated checkpoint vector"; return false; }
    return true;
}
}  // namespace

void save_checkpoint_file(const std::string& path, const wlg_snapshot& s, uint64_t n, uint64_t bins) {
    const std::string temporary = path + ".tmp";
    {
        std::ofstream out(temporary, std::ios::binary | std::ios::trunc);
        if (!out) throw WlgError(WLG_ERR_IO, "Cannot write checkpoint " + temporary);
        const char magic[8] = {'W', 'L', 'C', 'H', 'K', 'P', '3', '\0'};
        out.write(magic, 8);
        put(out, s.walker_id);
        put_vec(out, s.spins, n);
        put_vec(out, s.fields, n);
        put(out, s.energy);
        put_vec(out, s.log_g, bins);
        put_vec(out, s.histogram, bins);
        put_vec(out, s.active, bins);
        put(out, s.factor);
        put(out, s.attempted);
        put(out, s.accepted);
        put(out, s.forced_accepted);
        put(out, s.last_accepted_attempt);
        put(out, s.stage);
        for (int k = 0; k < 4; ++k) put(out, s.rng_state[k]);
        out.close();
        if (!out) throw WlgError(WLG_ERR_IO, "Failed writing checkpoint");
    }
    std::error_code ec;
    std::filesystem::remove(path, ec);
    ec.clear();
    std::filesystem::rename(temporary, path, ec);
    if (ec) throw WlgError(WLG_ERR_IO, "Cannot atomically replace checkpoint: " + ec.message());
}

bool load_checkpoint_file(const std::string& path, std::vector<int8_t>& spins, std::vector<double>& fields,
                          std::vector<double>& log_g, std::vector<uint64_t>& hist, std::vector<uint8_t>& active,
                          wlg_snapshot& s, std::string& error) {
    std::ifstream in(path, std::ios::binary);
    if (!in) { error = "Cannot open checkpoint " + path; return false; }
    char magic[8] = {};
    in.read(magic, 8);
    const std::string version(magic, 7);
    if (!in || (version != "WLCHKP1" && version != "WLCHKP2" && version != "WLCHKP3")) {
        error = "Invalid checkpoint format";
        return false;
    }
    s = wlg_snapshot{};
    if (!get(in, s.walker_id)) { error = "Truncated checkpoint"; return false; }
    if (!get_vec(in, spins, error) || !get_vec(in, fields, error)) return false;
    if (!get(in, s.energy)) { error = "Truncated checkpoint"; return false; }
    if (!get_vec(in, log_g, error) || !get_vec(in, hist, error) || !get_vec(in, active, error)) return false;
    if (!get(in, s.factor) || !get(in, s.attempted) || !get(in, s.accepted)) { error = "Truncated checkpoint"; return false; }
    if (version == "WLCHKP3" && !get(in, s.forced_accepted)) { error = "Truncated checkpoint"; return false; }
    if (version == "WLCHKP2" || version == "WLCHKP3") {
        if (!get(in, s.last_accepted_attempt)) { error = "Truncated checkpoint"; return false; }
    } else {
        s.last_accepted_attempt = s.accepted == 0 ? 0 : s.attempted;
    }
    if (!get(in, s.stage)) { error = "Truncated checkpoint"; return false; }
    for (int k = 0; k < 4; ++k)
        if (!get(in, s.rng_state[k])) { error = "Truncated checkpoint"; return false; }
    return true;
}

}  // namespace wlg
