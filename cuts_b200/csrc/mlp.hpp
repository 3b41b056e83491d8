// mlp.hpp -- FP32 MLP cost model for the learned matching order.
#pragma once
#include <cstdint>

#include "host.hpp"

#define MLP_HIDDEN 64
#define MLP_MAX_IN 32

namespace cuts {

int mlp_param_count(int in);

// in -> 64 -> 64 -> 1 with ReLU, parameters resident on one GPU.
struct Mlp {
    int in = 0;
    int device = 0;
    float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
    float *d_scalar = nullptr;
    float *d_X = nullptr;  // staged samples: X rows, then targets / outputs
    int cap_rows = 0;
    int64_t step = 0;

    int create(int in_dim, uint64_t seed, int dev);
    void destroy();
    // mean squared error and its gradient w.r.t. every parameter
    int loss_grad(const float *X, const float *T, int n, float *loss, float *grad);
    // Adam over mini-batches of `batch` rows (0 = full batch) for `epochs`
    int train(const float *X, const float *T, int n, int epochs, int batch, float lr,
              float *final_loss);
    int predict(const float *X, int n, float *Y);
    int get_params(float *out);
    int set_params(const float *p);

  private:
    int upload(const float *X, const float *T, int n);
};

}  // namespace cuts
