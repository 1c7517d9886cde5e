// mlp.cu — the small multilayer perceptron of the learned warm start (no counterpart in the
// reference): fully connected layers, tanh on the hidden layers, identity output, mean
// squared error, full-batch Adam.  Forward, backward and the optimiser are hand-written
// FP32 kernels; the network has a few thousand parameters and batches of a few thousand
// (features -> log g per spin) points, so every kernel is a latency-bound sweep over a tile
// that stays in shared memory, and no tensor-core path is worth its set-up here.
//
// Parameters are one FP32 array: for layer l, W_l (dims[l+1] x dims[l], row-major) then
// b_l (dims[l+1]).  Gradients use the same layout.  All reductions are deterministic (no
// atomics on gradients): a gradient call returns the same bits on every run.
#include <cmath>
#include <memory>
#include <vector>

#include "engine.hpp"

namespace wlg {

namespace {

constexpr int kTile = 16;
constexpr int kMaxLayers = 8;

// A = act(X W^T + b): X is B x in, W is out x in, A is B x out.
__global__ void dense_forward_kernel(const float* __restrict__ X, const float* __restrict__ W,
                                     const float* __restrict__ bias, float* __restrict__ A, int B, int in, int out,
                                     int tanh_act) {
    __shared__ float xs[kTile][kTile + 1];
    __shared__ float ws[kTile][kTile + 1];
    const int r = blockIdx.y * kTile + threadIdx.y;  // batch row
    const int o = blockIdx.x * kTile + threadIdx.x;  // output unit
    float acc = 0.f;
    for (int k0 = 0; k0 < in; k0 += kTile) {
        const int kx = k0 + threadIdx.x;
        xs[threadIdx.y][threadIdx.x] = (r < B && kx < in) ? X[static_cast<size_t>(r) * in + kx] : 0.f;
        const int wo = blockIdx.x * kTile + threadIdx.y;
        ws[threadIdx.y][threadIdx.x] = (wo < out && kx < in) ? W[static_cast<size_t>(wo) * in + kx] : 0.f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kTile; ++k) acc = fmaf(xs[threadIdx.y][k], ws[threadIdx.x][k], acc);
        __syncthreads();
    }
    if (r < B && o < out) {
        const float z = acc + bias[o];
        A[static_cast<size_t>(r) * out + o] = tanh_act ? tanhf(z) : z;
    }
}

// dX = dZ W: dZ is B x out, W is out x in, dX is B x in.
__global__ void dense_backward_input_kernel(const float* __restrict__ dZ, const float* __restrict__ W,
                                            float* __restrict__ dX, int B, int in, int out) {
    __shared__ float zs[kTile][kTile + 1];
    __shared__ float ws[kTile][kTile + 1];
    const int r = blockIdx.y * kTile + threadIdx.y;
    const int i = blockIdx.x * kTile + threadIdx.x;
    float acc = 0.f;
    for (int o0 = 0; o0 < out; o0 += kTile) {
        const int oz = o0 + threadIdx.x;
        zs[threadIdx.y][threadIdx.x] = (r < B && oz < out) ? dZ[static_cast<size_t>(r) * out + oz] : 0.f;
        const int ow = o0 + threadIdx.y;
        ws[threadIdx.y][threadIdx.x] = (ow < out && i < in) ? W[static_cast<size_t>(ow) * in + i] : 0.f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kTile; ++k) acc = fmaf(zs[threadIdx.y][k], ws[k][threadIdx.x], acc);
        __syncthreads();
    }
    if (r < B && i < in) dX[static_cast<size_t>(r) * in + i] = acc;
}

// dW = dZ^T X (out x in) and db = column sums of dZ, summed over the batch in a fixed order.
__global__ void dense_backward_weight_kernel(const float* __restrict__ dZ, const float* __restrict__ X,
                                             float* __restrict__ dW, float* __restrict__ db, int B, int in,
                                             int out) {
    __shared__ float zs[kTile][kTile + 1];  // [row][o]
    __shared__ float xs[kTile][kTile + 1];  // [row][i]
    const int o = blockIdx.y * kTile + threadIdx.y;
    const int i = blockIdx.x * kTile + threadIdx.x;
    float acc = 0.f, bacc = 0.f;
    for (int r0 = 0; r0 < B; r0 += kTile) {
        const int rz = r0 + threadIdx.y;
        const int oz = blockIdx.y * kTile + threadIdx.x;
        zs[threadIdx.y][threadIdx.x] = (rz < B && oz < out) ? dZ[static_cast<size_t>(rz) * out + oz] : 0.f;
        xs[threadIdx.y][threadIdx.x] = (rz < B && i < in) ? X[static_cast<size_t>(rz) * in + i] : 0.f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kTile; ++k) {
            acc = fmaf(zs[k][threadIdx.y], xs[k][threadIdx.x], acc);
            bacc += zs[k][threadIdx.y];
        }
        __syncthreads();
    }
    if (o < out && i < in) dW[static_cast<size_t>(o) * in + i] = acc;
    if (o < out && blockIdx.x == 0 && threadIdx.x == 0) db[o] = bacc;
}

// dZ = dA * (1 - A^2) for tanh layers.
__global__ void tanh_backward_kernel(const float* __restrict__ dA, const float* __restrict__ A,
                                     float* __restrict__ dZ, size_t n) {
    const size_t k = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) dZ[k] = dA[k] * (1.f - A[k] * A[k]);
}

// dY = 2 (Y - T) / B; per-block partial sums of (Y - T)^2 / B in FP64.
__global__ void mse_kernel(const float* __restrict__ Y, const float* __restrict__ T, float* __restrict__ dY,
                           double* __restrict__ partial, int B) {
    __shared__ double red[256];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double e2 = 0.0;
    if (k < B) {
        const float d = Y[k] - T[k];
        dY[k] = 2.f * d / static_cast<float>(B);
        e2 = static_cast<double>(d) * static_cast<double>(d) / static_cast<double>(B);
    }
    red[threadIdx.x] = e2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void sum_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += partial[k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Adam (Kingma & Ba 2015) with bias correction.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float beta1, float beta2, float eps,
                            float c1, float c2) {
    const size_t k = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = beta1 * m[k] + (1.f - beta1) * gk;
    const float vk = beta2 * v[k] + (1.f - beta2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace

class Mlp {
  public:
    Mlp(int layers, const int32_t* dims, uint64_t seed) : layers_(layers) {
        if (layers < 1 || layers > kMaxLayers) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "1 to 8 layers");
        for (int l = 0; l <= layers; ++l) {
            if (dims[l] < 1 || dims[l] > 4096) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "layer widths 1 to 4096");
            dims_[l] = dims[l];
        }
        if (dims_[layers] != 1) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "the output layer has one unit");
        size_t at = 0;
        for (int l = 0; l < layers; ++l) {
            woff_[l] = at;
            at += static_cast<size_t>(dims_[l + 1]) * dims_[l];
            boff_[l] = at;
            at += static_cast<size_t>(dims_[l + 1]);
        }
        count_ = at;
        // Glorot-uniform weights, zero biases, from a splitmix64 stream
        std::vector<float> h(count_, 0.f);
        uint64_t x = seed;
        for (int l = 0; l < layers; ++l) {
            const double a = std::sqrt(6.0 / static_cast<double>(dims_[l] + dims_[l + 1]));
            for (size_t k = 0; k < static_cast<size_t>(dims_[l + 1]) * dims_[l]; ++k) {
                const double u = static_cast<double>(splitmix(x) >> 11) * 0x1.0p-53;
                h[woff_[l] + k] = static_cast<float>((2.0 * u - 1.0) * a);
            }
        }
        check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        params_.allocate(count_ * 4);
        grads_.allocate(count_ * 4);
        m_.allocate(count_ * 4);
        v_.allocate(count_ * 4);
        check_cuda(cudaMemcpyAsync(params_.ptr, h.data(), count_ * 4, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaMemsetAsync(m_.ptr, 0, count_ * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(v_.ptr, 0, count_ * 4, stream_), "memset");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }
    ~Mlp() {
        if (stream_) {
            cudaStreamSynchronize(stream_);
            cudaStreamDestroy(stream_);
        }
    }
    size_t count() const { return count_; }

    void get(float* out) {
        check_cuda(cudaMemcpyAsync(out, params_.ptr, count_ * 4, cudaMemcpyDeviceToHost, stream_), "copy");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }
    void set(const float* in) {
        check_cuda(cudaMemcpyAsync(params_.ptr, in, count_ * 4, cudaMemcpyHostToDevice, stream_), "copy");
        check_cuda(cudaMemsetAsync(m_.ptr, 0, count_ * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(v_.ptr, 0, count_ * 4, stream_), "memset");
        step_ = 0;
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }

    void forward(const float* x, uint64_t batch, float* y) {
        upload(x, nullptr, batch);
        run_forward();
        check_cuda(cudaMemcpyAsync(y, act_ptr(layers_), batch_ * 4, cudaMemcpyDeviceToHost, stream_), "copy");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }

    double gradients(const float* x, const float* t, uint64_t batch, float* g) {
        upload(x, t, batch);
        run_backward();
        if (g) check_cuda(cudaMemcpyAsync(g, grads_.ptr, count_ * 4, cudaMemcpyDeviceToHost, stream_), "copy");
        return read_loss();
    }

    double train(const float* x, const float* t, uint64_t batch, uint64_t steps, double lr) {
        upload(x, t, batch);
        for (uint64_t s = 0; s < steps; ++s) {
            run_backward();
            ++step_;
            const float c1 = 1.f - std::pow(0.9f, static_cast<float>(step_));
            const float c2 = 1.f - std::pow(0.999f, static_cast<float>(step_));
            adam_kernel<<<static_cast<unsigned>((count_ + 255) / 256), 256, 0, stream_>>>(
                params_.get<float>(), grads_.get<float>(), m_.get<float>(), v_.get<float>(), count_,
                static_cast<float>(lr), 0.9f, 0.999f, 1e-8f, c1, c2);
            check_cuda(cudaGetLastError(), "adam_kernel");
        }
        run_forward();
        loss_pass();
        return read_loss();
    }

  private:
    float* act_ptr(int l) { return acts_.get<float>() + aoff_[l]; }

    void upload(const float* x, const float* t, uint64_t batch) {
        if (batch == 0 || batch > (1u << 24)) throw WlgError(WLG_ERR_INVALID_ARGUMENT, "batch must be 1 to 2^24");
        batch_ = static_cast<int>(batch);
        size_t at = 0, widest = 0;
        for (int l = 0; l <= layers_; ++l) {
            aoff_[l] = at;
            at += batch * static_cast<size_t>(dims_[l]);
            widest = std::max(widest, static_cast<size_t>(dims_[l]));
        }
        if (acts_.bytes < at * 4) acts_.allocate(at * 4);
        if (da_.bytes < batch * widest * 4) {
            da_.allocate(batch * widest * 4);
            dz_.allocate(batch * widest * 4);
        }
        if (target_.bytes < batch * 4) target_.allocate(batch * 4);
        const size_t blocks = (batch + 255) / 256;
        if (partial_.bytes < blocks * 8 + 8) partial_.allocate(blocks * 8 + 8);
        check_cuda(cudaMemcpyAsync(act_ptr(0), x, batch * dims_[0] * 4, cudaMemcpyHostToDevice, stream_), "copy x");
        if (t) check_cuda(cudaMemcpyAsync(target_.ptr, t, batch * 4, cudaMemcpyHostToDevice, stream_), "copy t");
    }

    void run_forward() {
        const float* p = params_.get<float>();
        for (int l = 0; l < layers_; ++l) {
            const dim3 grid((dims_[l + 1] + kTile - 1) / kTile, (batch_ + kTile - 1) / kTile);
            dense_forward_kernel<<<grid, dim3(kTile, kTile), 0, stream_>>>(act_ptr(l), p + woff_[l], p + boff_[l],
                                                                           act_ptr(l + 1), batch_, dims_[l],
                                                                           dims_[l + 1], l + 1 < layers_ ? 1 : 0);
            check_cuda(cudaGetLastError(), "dense_forward_kernel");
        }
    }

    void loss_pass() {
        const int blocks = (batch_ + 255) / 256;
        double* part = partial_.get<double>();
        mse_kernel<<<blocks, 256, 0, stream_>>>(act_ptr(layers_), target_.get<float>(), dz_.get<float>(), part,
                                                batch_);
        sum_kernel<<<1, 256, 0, stream_>>>(part, blocks, part + blocks);
        check_cuda(cudaGetLastError(), "mse_kernel");
    }

    // Forward, loss and the gradient of every parameter into grads_ (the loss stays on the
    // device; read_loss fetches it).
    void run_backward() {
        run_forward();
        const int blocks = (batch_ + 255) / 256;
        double* part = partial_.get<double>();
        float* dz = dz_.get<float>();
        float* da = da_.get<float>();
        mse_kernel<<<blocks, 256, 0, stream_>>>(act_ptr(layers_), target_.get<float>(), dz, part, batch_);
        sum_kernel<<<1, 256, 0, stream_>>>(part, blocks, part + blocks);
        check_cuda(cudaGetLastError(), "mse_kernel");
        const float* p = params_.get<float>();
        float* g = grads_.get<float>();
        for (int l = layers_ - 1; l >= 0; --l) {
            // dz holds dL/dZ of layer l (the output layer is linear)
            const dim3 wgrid((dims_[l] + kTile - 1) / kTile, (dims_[l + 1] + kTile - 1) / kTile);
            dense_backward_weight_kernel<<<wgrid, dim3(kTile, kTile), 0, stream_>>>(
                dz, act_ptr(l), g + woff_[l], g + boff_[l], batch_, dims_[l], dims_[l + 1]);
            check_cuda(cudaGetLastError(), "dense_backward_weight_kernel");
            if (l == 0) break;
            const dim3 igrid((dims_[l] + kTile - 1) / kTile, (batch_ + kTile - 1) / kTile);
            dense_backward_input_kernel<<<igrid, dim3(kTile, kTile), 0, stream_>>>(dz, p + woff_[l], da, batch_,
                                                                                   dims_[l], dims_[l + 1]);
            check_cuda(cudaGetLastError(), "dense_backward_input_kernel");
            const size_t n = static_cast<size_t>(batch_) * dims_[l];
            tanh_backward_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream_>>>(da, act_ptr(l), dz, n);
            check_cuda(cudaGetLastError(), "tanh_backward_kernel");
        }
    }

    // The loss that the last run_backward or loss pass left on the device.
    double read_loss() {
        const int blocks = (batch_ + 255) / 256;
        double loss = 0.0;
        check_cuda(cudaMemcpyAsync(&loss, partial_.get<double>() + blocks, 8, cudaMemcpyDeviceToHost, stream_),
                   "copy");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        return loss;
    }

    int layers_;
    int dims_[kMaxLayers + 1] = {};
    size_t woff_[kMaxLayers] = {}, boff_[kMaxLayers] = {}, aoff_[kMaxLayers + 1] = {};
    size_t count_ = 0;
    int batch_ = 0;
    uint64_t step_ = 0;
    cudaStream_t stream_ = nullptr;
    DeviceBuffer params_, grads_, m_, v_, acts_, da_, dz_, target_, partial_;
};

Mlp* mlp_create(int layers, const int32_t* dims, uint64_t seed) { return new Mlp(layers, dims, seed); }
void mlp_destroy(Mlp* m) { delete m; }
size_t mlp_count(const Mlp* m) { return m->count(); }
void mlp_get(Mlp* m, float* out) { m->get(out); }
void mlp_set(Mlp* m, const float* in) { m->set(in); }
void mlp_forward(Mlp* m, const float* x, uint64_t batch, float* y) { m->forward(x, batch, y); }
double mlp_gradients(Mlp* m, const float* x, const float* t, uint64_t batch, float* g) {
    return m->gradients(x, t, batch, g);
}
double mlp_train(Mlp* m, const float* x, const float* t, uint64_t batch, uint64_t steps, double lr) {
    return m->train(x, t, batch, steps, lr);
}

}  // namespace wlg
