// Device state of the learned warm start (see mlp.cu for the network).  Internal.
#ifndef CLOTHSTEP_MLP_H
#define CLOTHSTEP_MLP_H

#include <cuda_bf16.h>

#include "cs_internal.h"

#define MLP_W1 0
#define MLP_B1 2048
#define MLP_W2 2112
#define MLP_B2 10304
#define MLP_W3 10368
#define MLP_B3 14464
#define MLP_W4 14528
#define MLP_B4 14720
#define MLP_P 14723
#define MLP_NSTAT 38  // mu[16], sigma[16], mu_y[3], sigma_y[3]

struct MlpDev {
    float* w = nullptr;           // MLP_P master weights (FP32)
    __nv_bfloat16* wb = nullptr;  // MLP_P BF16 copies (weights used by the kernels)
    float *m = nullptr, *v = nullptr;
    float* gpart = nullptr;       // grid x MLP_P per-CTA gradient partials
    float* loss_part = nullptr;   // grid
    float* stats = nullptr;       // MLP_NSTAT
    float* feat = nullptr;        // N x 16 raw features of the current system
    __nv_bfloat16* h1 = nullptr;  // N x 64
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr, *y = nullptr;  // training activations
    float* du2 = nullptr;         // N x 128 gradient w.r.t. u2
    float* dfeat = nullptr;       // dataset: slots x N x 16
    float* dtarget = nullptr;     // dataset: slots x N x 3 (dv - previous dv)
    // energy-norm training (cs_mlp_train_step / cs_mlp_energy_gradient)
    float* pred = nullptr;        // N x 3 predictions of the current minibatch
    float* dy = nullptr;          // N x 3 A pred
    double* epart = nullptr;      // per slice two FP64 partials
    double* sheet_c = nullptr;    // per sheet dv*^T b (the solution's energy)
    float* sheet_scale = nullptr; // per sheet the gradient's coefficients of A pred and of b
    float* sheet_loss = nullptr;  // per sheet sin^2 of the A-angle between pred and dv*
    int slots = 0, grid = 0;
    int* err = nullptr;           // set if a tensor-core wait gave up
};


__global__ void cs_mlp_features_kernel(Batch B, MlpDev M, float* out);
__global__ void cs_mlp_l1_kernel(Batch B, MlpDev M, const float* fsrc, int n0, int n1, float* z1);
__global__ void cs_mlp_l23_kernel(Batch B, MlpDev M, int n0, int n1, float* z2, float* z3, float* yout, float* pred);
__global__ void cs_mlp_bwd23_kernel(Batch B, MlpDev M, int n0, int n1, const float* target);
__global__ void cs_mlp_bwd1_kernel(Batch B, MlpDev M, const float* fsrc, int n0, int n1);
__global__ void cs_mlp_adam_kernel(MlpDev M, int ncta, float lr, float b1, float b2, float eps, int step,
                                   float* grad_out);
__global__ void cs_mlp_adam_ext_kernel(MlpDev M, const float* grad, float lr, float b1, float b2, float eps, int step);
__global__ void cs_mlp_target_kernel(Batch B, const float* feat, float* target);
__global__ void cs_mlp_moments_kernel(const float* feat, const float* target, long long n, double* out);
__global__ void cs_mlp_loss_acc_kernel(MlpDev M, int ncta, float* acc);
__global__ void cs_mlp_energy_kernel(Batch B, MlpDev M, int sl0, int sl1);
__global__ void cs_mlp_energy_norm_kernel(Batch B, MlpDev M, int sl0, int sl1);
__global__ void cs_mlp_energy_sheet_kernel(Batch B, MlpDev M, int s0, int s1, int mode);
__global__ void cs_mlp_energy_loss_kernel(MlpDev M, int s0, int s1, float* acc);

// dynamic shared memory of the tile kernels (bytes)
#define MLP_SMEM_L1 12816
#define MLP_SMEM_L23 51216
#define MLP_SMEM_BWD23 145232
#define MLP_SMEM_BWD1 50304

#endif
