#pragma once
#include "common.cuh"

// Learned smoothing-length predictor: MLP 12 -> 64 -> 64 -> 1 with SiLU,
// BF16 weights and activations on the tensor cores (mma.sync m16n8k16, FP32
// accumulation), FP32 master weights and Adam state.
//
// Parameter layout (floats, also the layout of mhpc_mlp_get/set_params):
//   W1 [64][16]  (output unit, input feature; inputs 12..15 are zero padding)
//   b1 [64]
//   W2 [64][64]  (output unit, input unit)
//   b2 [64]
//   w3 [64]
//   b3 [1]
#define MLP_IN 12
#define MLP_INP 16
#define MLP_H 64
#define MLP_OFF_W1 0
#define MLP_OFF_B1 (MLP_OFF_W1 + MLP_H * MLP_INP)
#define MLP_OFF_W2 (MLP_OFF_B1 + MLP_H)
#define MLP_OFF_B2 (MLP_OFF_W2 + MLP_H * MLP_H)
#define MLP_OFF_W3 (MLP_OFF_B2 + MLP_H)
#define MLP_OFF_B3 (MLP_OFF_W3 + MLP_H)
#define MLP_NPARAM (MLP_OFF_B3 + 1)

struct mhpc_ctx;
struct MlpState;

// Everything the feature / prediction kernel reads (sorted order unless noted).
struct MlpFeatureInputs {
    int n;
    const int* perm;           // sorted -> original index
    const double* h;           // converged h of this RHS
    const double* h_start;     // h the iteration started from (previous step's)
    const double* rho;
    const double* cs;
    const double *vx, *vy, *vz;
    const int* noi;
    const int* nit;            // iterations used (-1 if none)
    const double *ax, *ay, *az;        // original order (SPH acceleration)
    const double *gx, *gy, *gz;        // original order, may be null
    const double* drhodt;              // original order
    const double* m;
    double dt;
    int target;
};

int mlp_create(MlpState** out, int capacity);
void mlp_destroy(MlpState* m);
int mlp_reset(MlpState* m, unsigned long long seed, cudaStream_t s);
int mlp_train(MlpState* m, int iters, float lr, int batch, float* loss_out, cudaStream_t s);
// Once trained: `iters` more Adam steps on the pairs collected so far, queued
// on `s` without a host synchronisation (the normalisation stays that of the
// first training).  No-op before the first mlp_train.
int mlp_refresh(MlpState* m, int iters, float lr, int batch, cudaStream_t s);
int mlp_forward_backward(MlpState* m, const float* feats, int rows, const float* target, float* out, float* grad,
                         float* loss_out, cudaStream_t s);
int mlp_get_params(MlpState* m, float* host, cudaStream_t s);
int mlp_set_params(MlpState* m, const float* host, cudaStream_t s);
int mlp_ready(const MlpState* m);
int mlp_has_prediction(const MlpState* m);
// Replace the starting h (sorted) with the predicted one where a prediction exists.
int mlp_apply_prediction(MlpState* m, const int* perm, double* h_sorted, int n, cudaStream_t s);
// Add (features of the previous RHS, log(h_new / h_start)) pairs to the training buffer.
int mlp_collect(MlpState* m, const int* perm, const double* h_start, const double* h_new, const int* count,
                const int* nit, int target, int tol, int max_iter, int n, cudaStream_t s);
// Features of this RHS (stored for the next collection) and, once trained,
// the predicted h of the next RHS.
int mlp_features_predict(MlpState* m, const MlpFeatureInputs& in, cudaStream_t s);
