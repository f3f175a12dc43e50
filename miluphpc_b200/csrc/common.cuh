// Internal definitions shared by the CUDA translation units of libmhpc.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mhpc.h"

#define MHPC_MAX_LEVEL 21
#define MHPC_WARP 32
#define MHPC_FULL 0xffffffffu

// Device status word: the first nonzero code wins; detail records the
// offending index; counters collect per-RHS statistics.
struct DevStatus {
    int code;
    int detail;
    int key_collisions;
    int max_level;
    int max_noi;
    int timeout_site;
    unsigned long long interactions;
    unsigned long long nodes_visited;
    unsigned long long noi_sum;
    int sml_out_of_band;
    int predictor_used;
    int predictor_fallback;
    int sml_unconverged;
    unsigned long long quad_interactions;  // accepted cells with a quadrupole term
    int sml_band_before;                   // out-of-band particles before the band repair
    int sml_band_skipped;                  // band repair rounds skipped (event buffer full)
    int pad[2];
};

// Device-side totals of the per-RHS counters over a run (mhpc_stats run_*).
struct RunTotals {
    unsigned long long rhs, oob_sum, oob_max, before_sum, band_rhs, used_sum, fallback_sum, pad;
};

__device__ __forceinline__ void set_status(DevStatus* st, int code, int detail) {
    if (atomicCAS(&st->code, 0, code) == 0) st->detail = detail;
}

#define CUDA_TRY(expr)                                  \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return MHPC_ERR_CUDA;    \
    } while (0)

static inline int grid_for(long n, int block, int cap = 148 * 32) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

__device__ __forceinline__ double4 ldg_d4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Ordered-integer encoding of doubles for atomicMin/atomicMax.
__device__ __forceinline__ long long dbl_to_ord(double v) {
    long long b = __double_as_longlong(v);
    return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}
__host__ __device__ __forceinline__ double ord_to_dbl(long long o) {
    long long b = o >= 0 ? o : (o ^ 0x7fffffffffffffffLL);
#ifdef __CUDA_ARCH__
    return __longlong_as_double(b);
#else
    union { long long l; double d; } u;
    u.l = b;
    return u.d;
#endif
}

// ---------------------------------------------------------------- sort
size_t sort_scratch_bytes(int n);
int sort_pairs_u64(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out, int* vals_out,
                   int n, void* scratch, size_t scratch_bytes, DevStatus* st, cudaStream_t s);

// ---------------------------------------------------------------- scan
size_t scan_scratch_bytes(int n);
// Exclusive scan of n ints into out (n+1 entries, out[n] = total).
int scan_exclusive_i32(const int* in, int* out, int n, void* scratch, cudaStream_t s);

// ---------------------------------------------------------------- keys
int launch_bbox(const double* x, const double* y, const double* z, int n, long long* ord_minmax,
                DevStatus* st, cudaStream_t s);
int launch_bbox_finish(const long long* ord_minmax, double* bbox6, cudaStream_t s);
int launch_keys(const double* x, const double* y, const double* z, int n, const long long* ord_minmax,
                int curve, uint64_t* keys, int* iota, cudaStream_t s);
// keys from a caller-provided cubic box (6 doubles on the device)
int launch_keys_box(const double* x, const double* y, const double* z, int n, const double* bbox, int curve,
                    uint64_t* keys, cudaStream_t s);
