// Learned smoothing-length predictor (placeholder until the tensor-core
// kernels land): every entry point reports MHPC_ERR_UNSUPPORTED.
#include "mlp.cuh"

struct MlpState {
    int capacity;
};

int mlp_create(MlpState** out, int capacity) {
    (void)capacity;
    *out = nullptr;
    return MHPC_ERR_UNSUPPORTED;
}
void mlp_destroy(MlpState* m) { delete m; }
int mlp_predict_h(MlpState*, mhpc_ctx*, int) { return MHPC_ERR_UNSUPPORTED; }
int mlp_collect(MlpState*, mhpc_ctx*, int) { return MHPC_ERR_UNSUPPORTED; }

extern "C" {
int mhpc_mlp_reset(mhpc_ctx*, uint64_t) { return MHPC_ERR_UNSUPPORTED; }
int mhpc_mlp_train(mhpc_ctx*, int, float, float*) { return MHPC_ERR_UNSUPPORTED; }
int mhpc_mlp_num_params(void) { return 12 * 64 + 64 + 64 * 64 + 64 + 64 + 1; }
int mhpc_mlp_forward_backward(mhpc_ctx*, const float*, int, const float*, float*, float*, float*) {
    return MHPC_ERR_UNSUPPORTED;
}
int mhpc_mlp_get_params(mhpc_ctx*, float*) { return MHPC_ERR_UNSUPPORTED; }
int mhpc_mlp_set_params(mhpc_ctx*, const float*) { return MHPC_ERR_UNSUPPORTED; }
}
