// Learned warm start: a pair-wise MLP that proposes the start of the BPSDP
// iteration from the active-space integrals.  No counterpart in the
// reference, whose start is the random guess of Guess() (v2rdm_solver.cc:
// 2386-2516).
//
// For every orbital pair p <= q of an all-active C1 singlet the network reads
// kWsFeatures numbers computed from h and the three-index integrals (one- and
// two-electron integrals of the pair, their ranks and the filling) and
// proposes three: the alpha 1-RDM element gamma_pq, the D2ab pair diagonal
// D2ab(pq,pq) and a contribution to log(mu).  Four dense layers
// (kWsFeatures -> H -> H -> H -> 3, ReLU), BF16 weights with FP32 arithmetic
// (mlp.cu); training keeps FP32 master weights and runs Adam on the mean
// squared error against converged solutions this solver produced.  The
// proposal becomes x0 (D1, Q1 = 1 - D1 and the D2ab diagonal; everything else
// zero), which the solve projects onto A x = b with its own CG (start = 2),
// with zero duals and mu from the network.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>
#include <vector>

#include "kernels.cuh"
#include "mlp.h"
#include "warmstart.h"

namespace v2g {

namespace {

#define WCK(call)                                                                                          \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() {
        if (p) cudaFree(p);
    }
    void ensure(size_t count) {
        if (count <= n) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        WCK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
};

}  // namespace

struct WsNet {
    int H = 0, device = 0;
    int dims[kWsLayers + 1];  // in, H, H, H, out
    std::vector<int64_t> woff, boff;
    int64_t nparams = 0;
    Buf<float> w, m, v, g;
    Buf<__nv_bfloat16> w16;
    // activations of the last forward pass: act[0] = input rows, act[l + 1] = layer l's output
    Buf<float> act[kWsLayers + 1], dact[2], targ, delta;
    Buf<double> partial;
    int64_t rows_cap = 0;
    int step = 0;
    cudaStream_t s = nullptr;

    WsNet(int hidden, int dev, unsigned long long seed) : H(hidden), device(dev) {
        dims[0] = kWsFeatures;
        for (int l = 1; l < kWsLayers; l++) dims[l] = H;
        dims[kWsLayers] = kWsOut;
        for (int l = 0; l < kWsLayers; l++) {
            woff.push_back(nparams);
            nparams += (int64_t)dims[l + 1] * dims[l];
            boff.push_back(nparams);
            nparams += dims[l + 1];
        }
        WCK(cudaSetDevice(device));
        WCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        w.ensure(nparams);
        m.ensure(nparams);
        v.ensure(nparams);
        g.ensure(nparams);
        w16.ensure(nparams);
        // He initialisation for the ReLU layers, zero biases
        std::mt19937_64 rng(seed);
        std::vector<float> hw(nparams, 0.f);
        for (int l = 0; l < kWsLayers; l++) {
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / dims[l]) * (l + 1 == kWsLayers ? 0.1f : 1.f));
            for (int64_t i = 0; i < (int64_t)dims[l + 1] * dims[l]; i++) hw[woff[l] + i] = nd(rng);
        }
        set_params(hw.data());
    }
    ~WsNet() {
        if (s) cudaStreamDestroy(s);
    }
    void set_params(const float* hw) {
        WCK(cudaMemcpy(w.p, hw, nparams * sizeof(float), cudaMemcpyHostToDevice));
        WCK(cudaMemset(m.p, 0, nparams * sizeof(float)));
        WCK(cudaMemset(v.p, 0, nparams * sizeof(float)));
        mlp_to_bf16(nparams, w.p, w16.p, s);
        WCK(cudaStreamSynchronize(s));
        step = 0;
    }
    void reserve(int64_t rows) {
        if (rows <= rows_cap) return;
        for (int l = 0; l <= kWsLayers; l++) act[l].ensure((size_t)rows * dims[l]);
        dact[0].ensure((size_t)rows * H);
        dact[1].ensure((size_t)rows * H);
        targ.ensure((size_t)rows * kWsOut);
        delta.ensure((size_t)rows * kWsOut);
        partial.ensure(mlp_mse_blocks());
        rows_cap = rows;
    }
    // act[kWsLayers] = network(act[0]) for `rows` rows
    void forward(int rows) {
        for (int l = 0; l < kWsLayers; l++)
            mlp_gemm_bf16(rows, dims[l + 1], dims[l], act[l].p, dims[l], false, w16.p + woff[l], dims[l], true,
                          w.p + boff[l], l + 1 < kWsLayers, false, act[l + 1].p, dims[l + 1], s);
    }
    // g = d(mean squared error)/d(params) for the last forward pass against
    // targ; returns the loss (mean over rows and outputs)
    double backward(int rows) {
        const int64_t nout = (int64_t)rows * kWsOut;
        mlp_mse(nout, act[kWsLayers].p, targ.p, 1.f / (float)nout, delta.p, partial.p, s);
        const float* dy = delta.p;
        int cur = 0;
        for (int l = kWsLayers - 1; l >= 0; l--) {
            const int out = dims[l + 1], in = dims[l];
            // dW_l = dY^T act_l (out x in), db_l = column sums of dY
            mlp_gemm(out, in, rows, dy, out, true, act[l].p, in, false, nullptr, false, false, g.p + woff[l], in, s);
            mlp_col_sum(rows, out, dy, g.p + boff[l], s);
            if (l == 0) break;
            // dX = dY W_l, then through the ReLU of layer l - 1
            float* dx = dact[cur].p;
            mlp_gemm_bf16(rows, in, out, dy, out, false, w16.p + woff[l], in, false, nullptr, false, false, dx, in,
                          s);
            mlp_relu_back((int64_t)rows * in, act[l].p, dx, s);
            dy = dx;
            cur ^= 1;
        }
        std::vector<double> hp(mlp_mse_blocks());
        WCK(cudaMemcpyAsync(hp.data(), partial.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        WCK(cudaStreamSynchronize(s));
        double loss = 0.0;
        for (double v2 : hp) loss += v2;
        return loss / (double)nout;
    }
};

// Features of the pairs p <= q (row r of the output per pair, in the order
// p = 0..n-1, q = p..n-1), from h (n x n) and L (nq x n x n), all symmetric.
void ws_features(int n, double nalpha, const double* h, const double* L, int nq, float* out) {
    std::vector<double> J(n * n, 0.0), K(n * n, 0.0), X(n * n, 0.0);
    for (int Q = 0; Q < nq; Q++) {
        const double* l = L + (size_t)Q * n * n;
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++) {
                J[p * n + q] += l[p * n + p] * l[q * n + q];  // (pp|qq)
                K[p * n + q] += l[p * n + q] * l[p * n + q];  // (pq|pq)
            }
    }
    // sum_r (pr|qr) / n
    for (int Q = 0; Q < nq; Q++) {
        const double* l = L + (size_t)Q * n * n;
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++) {
                double t = 0.0;
                for (int r = 0; r < n; r++) t += l[p * n + r] * l[q * n + r];
                X[p * n + q] += t / n;
            }
    }
    double scale = 0.0;
    for (int p = 0; p < n; p++) scale = std::max(scale, std::fabs(h[p * n + p]));
    for (int p = 0; p < n; p++) scale = std::max(scale, J[p * n + p]);
    if (!(scale > 0.0)) scale = 1.0;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h[a * n + a] < h[b * n + b]; });
    std::vector<double> rank(n);
    for (int i = 0; i < n; i++) rank[order[i]] = i;
    const double den = n > 1 ? (double)(n - 1) : 1.0;
    int r = 0;
    for (int p = 0; p < n; p++)
        for (int q = p; q < n; q++, r++) {
            float* f = out + (size_t)r * kWsFeatures;
            f[0] = (float)(h[p * n + p] / scale);
            f[1] = (float)(h[q * n + q] / scale);
            f[2] = (float)(h[p * n + q] / scale);
            f[3] = (float)(J[p * n + q] / scale);
            f[4] = (float)(K[p * n + q] / scale);
            f[5] = (float)(J[p * n + p] / scale);
            f[6] = (float)(J[q * n + q] / scale);
            f[7] = p == q ? 1.f : 0.f;
            f[8] = (float)(rank[p] / den);
            f[9] = (float)(rank[q] / den);
            f[10] = (float)(nalpha / n);
            f[11] = (float)((rank[p] + 0.5 - nalpha) / n);
            f[12] = (float)((rank[q] + 0.5 - nalpha) / n);
            f[13] = (float)(X[p * n + q] / scale);
            f[14] = (float)(n / 24.0);
            f[15] = 1.f;
        }
}

}  // namespace v2g

using v2g::WsNet;

struct v2g_warmstart {
    WsNet net;
    v2g_warmstart(int hidden, int device, unsigned long long seed) : net(hidden, device, seed) {}
};

namespace v2g {

WsNet& ws_net(v2g_warmstart* w) { return w->net; }

int ws_create(int hidden, int device, unsigned long long seed, v2g_warmstart** out) {
    *out = new v2g_warmstart(hidden, device, seed);
    return 0;
}
void ws_destroy(v2g_warmstart* w) { delete w; }
int64_t ws_num_params(const v2g_warmstart* w) { return w->net.nparams; }

void ws_get_params(const v2g_warmstart* w, float* p) {
    WCK(cudaMemcpy(p, w->net.w.p, w->net.nparams * sizeof(float), cudaMemcpyDeviceToHost));
}
void ws_set_params(v2g_warmstart* w, const float* p) { w->net.set_params(p); }

void ws_forward(v2g_warmstart* w, int64_t rows, const float* feat, float* out) {
    WsNet& N = w->net;
    WCK(cudaSetDevice(N.device));
    N.reserve(rows);
    WCK(cudaMemcpyAsync(N.act[0].p, feat, rows * kWsFeatures * sizeof(float), cudaMemcpyHostToDevice, N.s));
    N.forward((int)rows);
    WCK(cudaMemcpyAsync(out, N.act[kWsLayers].p, rows * kWsOut * sizeof(float), cudaMemcpyDeviceToHost, N.s));
    WCK(cudaStreamSynchronize(N.s));
}

double ws_gradient(v2g_warmstart* w, int64_t rows, const float* feat, const float* targ, float* grad) {
    WsNet& N = w->net;
    WCK(cudaSetDevice(N.device));
    N.reserve(rows);
    WCK(cudaMemcpyAsync(N.act[0].p, feat, rows * kWsFeatures * sizeof(float), cudaMemcpyHostToDevice, N.s));
    WCK(cudaMemcpyAsync(N.targ.p, targ, rows * kWsOut * sizeof(float), cudaMemcpyHostToDevice, N.s));
    N.forward((int)rows);
    const double loss = N.backward((int)rows);
    if (grad) {
        WCK(cudaMemcpyAsync(grad, N.g.p, N.nparams * sizeof(float), cudaMemcpyDeviceToHost, N.s));
        WCK(cudaStreamSynchronize(N.s));
    }
    return loss;
}

// Adam over minibatches of the data set (rows in the given order, which the
// caller shuffles), `epochs` passes; the whole set lives on the device.
double ws_train(v2g_warmstart* w, int64_t rows, const float* feat, const float* targ, int epochs, int batch,
                float lr) {
    WsNet& N = w->net;
    WCK(cudaSetDevice(N.device));
    Buf<float> df, dt;
    df.ensure((size_t)rows * kWsFeatures);
    dt.ensure((size_t)rows * kWsOut);
    WCK(cudaMemcpyAsync(df.p, feat, rows * kWsFeatures * sizeof(float), cudaMemcpyHostToDevice, N.s));
    WCK(cudaMemcpyAsync(dt.p, targ, rows * kWsOut * sizeof(float), cudaMemcpyHostToDevice, N.s));
    N.reserve(batch);
    double last = 0.0;
    for (int e = 0; e < epochs; e++) {
        double sum = 0.0;
        int64_t cnt = 0;
        for (int64_t r0 = 0; r0 < rows; r0 += batch) {
            const int b = (int)std::min<int64_t>(batch, rows - r0);
            WCK(cudaMemcpyAsync(N.act[0].p, df.p + r0 * kWsFeatures, (size_t)b * kWsFeatures * sizeof(float),
                                cudaMemcpyDeviceToDevice, N.s));
            WCK(cudaMemcpyAsync(N.targ.p, dt.p + r0 * kWsOut, (size_t)b * kWsOut * sizeof(float),
                                cudaMemcpyDeviceToDevice, N.s));
            N.forward(b);
            const double loss = N.backward(b);
            mlp_adam(N.nparams, N.w.p, N.g.p, N.m.p, N.v.p, N.w16.p, lr, ++N.step, N.s);
            sum += loss * b;
            cnt += b;
        }
        last = sum / (double)cnt;
    }
    WCK(cudaStreamSynchronize(N.s));
    return last;
}

}  // namespace v2g
