// The learned warm start's network (warmstart.cu); the C ABI lives in solver.cu.
#pragma once

#include <cstdint>

struct v2g_warmstart;

namespace v2g {

constexpr int kWsFeatures = 16;  // per orbital pair
constexpr int kWsOut = 3;        // gamma_pq, D2ab(pq,pq), log(mu) contribution
constexpr int kWsLayers = 4;     // dense layers (three hidden ReLU layers)

int ws_create(int hidden, int device, unsigned long long seed, v2g_warmstart** out);
void ws_destroy(v2g_warmstart* w);
int64_t ws_num_params(const v2g_warmstart* w);
void ws_get_params(const v2g_warmstart* w, float* p);
void ws_set_params(v2g_warmstart* w, const float* p);
// pair features of an all-active space: n (n + 1) / 2 rows of kWsFeatures
void ws_features(int n, double nalpha, const double* h, const double* L, int nq, float* out);
void ws_forward(v2g_warmstart* w, int64_t rows, const float* feat, float* out);
double ws_gradient(v2g_warmstart* w, int64_t rows, const float* feat, const float* targ, float* grad);
double ws_train(v2g_warmstart* w, int64_t rows, const float* feat, const float* targ, int epochs, int batch, float lr);

}  // namespace v2g
