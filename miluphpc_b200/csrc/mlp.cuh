#pragma once
#include "common.cuh"

struct mhpc_ctx;
struct MlpState;

int mlp_create(MlpState** out, int capacity);
void mlp_destroy(MlpState* m);
// Predict h for every sorted particle from the features of the previous step
// and pre-mark particles whose predicted h lands in the neighbour band.
int mlp_predict_h(MlpState* m, mhpc_ctx* c, int n);
// Collect (features, converged h) pairs after a plain variable-h iteration.
int mlp_collect(MlpState* m, mhpc_ctx* c, int n);
