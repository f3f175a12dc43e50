// Learned smoothing-length predictor (not in the reference).
//
// A small MLP (12 -> 64 -> 64 -> 1, SiLU) predicts log(h_next / h) from
// per-particle features of the previous right-hand side.  Forward and
// backward passes run on the tensor cores with mma.sync.m16n8k16 (BF16
// operands, FP32 accumulation); master weights and Adam moments are FP32.
// The matrices are tiny (K = 16 or 64, N = 64, batch rows in tiles of 32), so
// one warp owns 32 rows end to end and the layer-to-layer hand-off stays in
// registers (the FP32 accumulator fragment of one mma is exactly the BF16 A
// fragment of the next).  Weight gradients over the batch are second mma
// passes on transposed copies in shared memory.
//
// Training data are (features of RHS k, log(h converged at RHS k+1 / h_k))
// pairs collected from the plain variable-h iteration.  Once trained, the
// prediction for RHS k+1 is made at the end of RHS k (with the features) and
// replaces the starting h of the iteration; particles whose predicted h lands
// in the neighbour band stop after the first sweep, the others continue the
// plain iteration (fallback).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "mlp.cuh"

struct MlpState {
    int cap = 0;
    float* feats = nullptr;     // [cap][MLP_IN], original order, features of the last RHS
    float* hlog = nullptr;      // [cap] predicted log(h_next / h), original order
    double* hbase = nullptr;    // [cap] h of the last RHS (original order), base of the prediction
    int have_feats = 0;
    int have_pred = 0;
    int trained = 0;
    int step = 0;
    float* w = nullptr;         // [MLP_NPARAM] FP32 master weights
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* grad = nullptr;
    __nv_bfloat16* w1t = nullptr;  // [64][16]
    __nv_bfloat16* w2t = nullptr;  // [64][64] (out, in)
    __nv_bfloat16* w2k = nullptr;  // [64][64] (in, out) for the backward product
    float* norm = nullptr;      // mean[12], inv_std[12], y_mean, y_std
    double* nsum = nullptr;     // 26 sums for the statistics
    float* loss = nullptr;
    int tcap = 0;
    float* tx = nullptr;        // [tcap][MLP_IN]
    float* ty = nullptr;        // [tcap]
    unsigned long long* tcount = nullptr;  // total pairs written (ring buffer)
    int adam_t = 0;
    std::vector<void*> allocs;
};

namespace {

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned*>(&v);
}

__device__ __forceinline__ void mma16816(float* d, const unsigned* a, const unsigned* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float silu(float x) { return x / (1.f + __expf(-x)); }
__device__ __forceinline__ float dsilu(float x) {
    const float s = 1.f / (1.f + __expf(-x));
    return s * (1.f + x * (1.f - s));
}

__device__ __forceinline__ unsigned ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const unsigned*>(p); }

// Shared-memory copy of the network for one block.
struct MlpSmem {
    __nv_bfloat16 w1t[MLP_H][MLP_INP];
    __nv_bfloat16 w2t[MLP_H][MLP_H];
    __nv_bfloat16 w2k[MLP_H][MLP_H];
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], b3;
    float norm[2 * MLP_IN + 2];
};

__device__ void load_net(MlpSmem& S, const __nv_bfloat16* w1t, const __nv_bfloat16* w2t, const __nv_bfloat16* w2k,
                         const float* w, const float* norm) {
    for (int i = threadIdx.x; i < MLP_H * MLP_INP; i += blockDim.x) (&S.w1t[0][0])[i] = w1t[i];
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) {
        (&S.w2t[0][0])[i] = w2t[i];
        (&S.w2k[0][0])[i] = w2k[i];
    }
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        S.b1[i] = w[MLP_OFF_B1 + i];
        S.b2[i] = w[MLP_OFF_B2 + i];
        S.w3[i] = w[MLP_OFF_W3 + i];
    }
    if (threadIdx.x == 0) S.b3 = w[MLP_OFF_B3];
    for (int i = threadIdx.x; i < 2 * MLP_IN + 2; i += blockDim.x) S.norm[i] = norm[i];
}

// Forward pass of 32 rows held by one warp.  xs: the warp's 32 x 16 BF16
// inputs in shared memory (row-major).  Returns, per lane, the output of row
// `lane`.  If h1/h2 are given, the pre-activations are kept (C fragments:
// [mt][nt][4]) for the backward pass and a1 receives the BF16 A fragments of
// the second layer ([mt][kk][4]).
struct Frags {
    float h1[2][8][4];
    float h2[2][8][4];
    unsigned a1[2][4][4];
};

__device__ float warp_forward(const MlpSmem& S, const __nv_bfloat16 (*xs)[MLP_INP], Frags& F) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // layer 1: [32 x 16] x [16 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        unsigned a[4];
        a[0] = ld32(&xs[mt * 16 + g][t * 2]);
        a[1] = ld32(&xs[mt * 16 + g + 8][t * 2]);
        a[2] = ld32(&xs[mt * 16 + g][t * 2 + 8]);
        a[3] = ld32(&xs[mt * 16 + g + 8][t * 2 + 8]);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            unsigned b[2];
            b[0] = ld32(&S.w1t[nt * 8 + g][t * 2]);
            b[1] = ld32(&S.w1t[nt * 8 + g][t * 2 + 8]);
            float* d = F.h1[mt][nt];
            const float bb0 = S.b1[nt * 8 + t * 2], bb1 = S.b1[nt * 8 + t * 2 + 1];
            d[0] = bb0; d[1] = bb1; d[2] = bb0; d[3] = bb1;
            mma16816(d, a, b);
        }
    }
    // SiLU -> BF16 A fragments of layer 2 (C layout of n-tiles 2kk, 2kk+1 = A layout of k-step kk)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const float* c0 = F.h1[mt][2 * kk];
            const float* c1 = F.h1[mt][2 * kk + 1];
            F.a1[mt][kk][0] = pack_bf16(silu(c0[0]), silu(c0[1]));
            F.a1[mt][kk][1] = pack_bf16(silu(c0[2]), silu(c0[3]));
            F.a1[mt][kk][2] = pack_bf16(silu(c1[0]), silu(c1[1]));
            F.a1[mt][kk][3] = pack_bf16(silu(c1[2]), silu(c1[3]));
        }
    // layer 2: [32 x 64] x [64 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float* d = F.h2[mt][nt];
            const float bb0 = S.b2[nt * 8 + t * 2], bb1 = S.b2[nt * 8 + t * 2 + 1];
            d[0] = bb0; d[1] = bb1; d[2] = bb0; d[3] = bb1;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                unsigned b[2];
                b[0] = ld32(&S.w2t[nt * 8 + g][kk * 16 + t * 2]);
                b[1] = ld32(&S.w2t[nt * 8 + g][kk * 16 + t * 2 + 8]);
                mma16816(d, F.a1[mt][kk], b);
            }
        }
    // output layer in FP32: rows g, g+8 of each m-tile, reduced over the quad
    float o[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float w0 = S.w3[nt * 8 + t * 2], w1 = S.w3[nt * 8 + t * 2 + 1];
            s0 += silu(F.h2[mt][nt][0]) * w0 + silu(F.h2[mt][nt][1]) * w1;
            s1 += silu(F.h2[mt][nt][2]) * w0 + silu(F.h2[mt][nt][3]) * w1;
        }
        s0 += __shfl_xor_sync(MHPC_FULL, s0, 1);
        s0 += __shfl_xor_sync(MHPC_FULL, s0, 2);
        s1 += __shfl_xor_sync(MHPC_FULL, s1, 1);
        s1 += __shfl_xor_sync(MHPC_FULL, s1, 2);
        o[mt][0] = s0 + S.b3;
        o[mt][1] = s1 + S.b3;
    }
    // row r = mt*16 + half*8 + g lives in quad g: fetch row `lane`
    const int mt = lane >> 4, half = (lane >> 3) & 1, src = (lane & 7) * 4;
    const float v00 = __shfl_sync(MHPC_FULL, o[0][0], src), v01 = __shfl_sync(MHPC_FULL, o[0][1], src);
    const float v10 = __shfl_sync(MHPC_FULL, o[1][0], src), v11 = __shfl_sync(MHPC_FULL, o[1][1], src);
    return mt == 0 ? (half ? v01 : v00) : (half ? v11 : v10);
}

// ----------------------------------------------------------- training step
constexpr int kTrainRows = 128;  // rows per block (4 warps x 32)

struct TrainSmem {
    MlpSmem net;
    __nv_bfloat16 xs[kTrainRows][MLP_INP];
    __nv_bfloat16 xt[MLP_INP][kTrainRows];
    __nv_bfloat16 a1t[MLP_H][kTrainRows];
    __nv_bfloat16 dh2t[MLP_H][kTrainRows];
    __nv_bfloat16 dh1t[MLP_H][kTrainRows];
    float db1[MLP_H], db2[MLP_H], dw3[MLP_H];
    float db3, loss;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// rows: explicit (feats/target of `rows` rows) or sampled from the ring
// buffer (count entries, cap tcap) with the seed.  Adds gradients of the
// mean-squared loss (scaled by 1/total_rows) into grad, loss into *loss, and
// writes the raw network outputs to out when given.
__global__ void __launch_bounds__(kTrainRows) k_train(const float* __restrict__ feats, const float* __restrict__ target,
                                                      int rows, const unsigned long long* tcount, int tcap,
                                                      unsigned long long seed, const float* __restrict__ w,
                                                      const __nv_bfloat16* w1t, const __nv_bfloat16* w2t,
                                                      const __nv_bfloat16* w2k, const float* norm, int normalise,
                                                      float* grad, float* loss, float* out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    load_net(S.net, w1t, w2t, w2k, w, norm);
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) { S.db1[i] = 0.f; S.db2[i] = 0.f; S.dw3[i] = 0.f; }
    if (threadIdx.x == 0) { S.db3 = 0.f; S.loss = 0.f; }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int r = threadIdx.x;                      // local row
    const long row = (long)blockIdx.x * kTrainRows + r;
    const bool valid = row < rows;
    // gather this row's features (sampled or explicit), normalise, BF16
    long src = row;
    if (!feats && tcount) {
        const unsigned long long cnt = *tcount;
        const unsigned long long avail = cnt < (unsigned long long)tcap ? cnt : (unsigned long long)tcap;
        src = avail ? (long)(mix64(seed * 0x100000001b3ULL + row) % avail) : 0;
    }
    const float* X = feats ? feats : nullptr;
    float y = 0.f;
    float xv[MLP_INP];
#pragma unroll
    for (int k = 0; k < MLP_INP; ++k) xv[k] = 0.f;
    if (valid) {
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) {
            float v = X[src * MLP_IN + k];
            if (normalise) v = (v - S.net.norm[k]) * S.net.norm[MLP_IN + k];
            xv[k] = v;
        }
        y = target[src];
        if (normalise) y = (y - S.net.norm[2 * MLP_IN]) / S.net.norm[2 * MLP_IN + 1];
    }
#pragma unroll
    for (int k = 0; k < MLP_INP; ++k) {
        const __nv_bfloat16 b = __float2bfloat16_rn(xv[k]);
        S.xs[r][k] = b;
        S.xt[k][r] = b;
    }
    __syncwarp();
    Frags F;
    const float o = warp_forward(S.net, &S.xs[warp * 32], F);
    const float scale = 1.f / (float)rows;
    const float diff = valid ? (o - y) : 0.f;
    const float dout = 2.f * diff * scale;
    if (out && valid) out[row] = o;
    float l2 = diff * diff * scale;
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) l2 += __shfl_xor_sync(MHPC_FULL, l2, q);
    float db3 = dout;
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) db3 += __shfl_xor_sync(MHPC_FULL, db3, q);
    if (lane == 0) { atomicAdd(&S.loss, l2); atomicAdd(&S.db3, db3); }
    // dout of rows g, g+8 of each m-tile
    float drow[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        drow[mt][0] = __shfl_sync(MHPC_FULL, dout, mt * 16 + g);
        drow[mt][1] = __shfl_sync(MHPC_FULL, dout, mt * 16 + g + 8);
    }
    // dH2 = dout w3 SiLU'(H2); dw3 = sum dout A2; A1^T to shared memory
    unsigned dh2a[2][4][4];
    float cs2[8][2], cw3[8][2];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) { cs2[nt][0] = cs2[nt][1] = 0.f; cw3[nt][0] = cw3[nt][1] = 0.f; }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        float d2[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = nt * 8 + t * 2 + (e & 1);
                const float h = F.h2[mt][nt][e];
                const float dr = drow[mt][e >> 1];
                d2[nt][e] = dr * S.net.w3[col] * dsilu(h);
                cw3[nt][e & 1] += dr * silu(h);
                cs2[nt][e & 1] += d2[nt][e];
                const int rloc = warp * 32 + mt * 16 + g + (e >> 1) * 8;
                S.dh2t[col][rloc] = __float2bfloat16_rn(d2[nt][e]);
            }
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            dh2a[mt][kk][0] = pack_bf16(d2[2 * kk][0], d2[2 * kk][1]);
            dh2a[mt][kk][1] = pack_bf16(d2[2 * kk][2], d2[2 * kk][3]);
            dh2a[mt][kk][2] = pack_bf16(d2[2 * kk + 1][0], d2[2 * kk + 1][1]);
            dh2a[mt][kk][3] = pack_bf16(d2[2 * kk + 1][2], d2[2 * kk + 1][3]);
            // A1 transposed (the BF16 values the forward used)
            const unsigned v[4] = {F.a1[mt][kk][0], F.a1[mt][kk][1], F.a1[mt][kk][2], F.a1[mt][kk][3]};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = kk * 16 + (e >> 1) * 8 + t * 2;
                const int rloc = warp * 32 + mt * 16 + g + (e & 1) * 8;
                const __nv_bfloat162 pr = *reinterpret_cast<const __nv_bfloat162*>(&v[e]);
                S.a1t[col][rloc] = pr.x;
                S.a1t[col + 1][rloc] = pr.y;
            }
        }
    }
    // column sums over the warp's rows -> shared
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            float a = cs2[nt][e], b = cw3[nt][e];
#pragma unroll
            for (int q = 4; q < 32; q <<= 1) {
                a += __shfl_xor_sync(MHPC_FULL, a, q);
                b += __shfl_xor_sync(MHPC_FULL, b, q);
            }
            if (g == 0) {
                atomicAdd(&S.db2[nt * 8 + t * 2 + e], a);
                atomicAdd(&S.dw3[nt * 8 + t * 2 + e], b);
            }
        }
    // dA1 = dH2 W2 (K = 64 outputs of layer 2), dH1 = dA1 SiLU'(H1)
    float cs1[8][2];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) cs1[nt][0] = cs1[nt][1] = 0.f;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                unsigned b[2];
                b[0] = ld32(&S.net.w2k[nt * 8 + g][kk * 16 + t * 2]);
                b[1] = ld32(&S.net.w2k[nt * 8 + g][kk * 16 + t * 2 + 8]);
                mma16816(d, dh2a[mt][kk], b);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = nt * 8 + t * 2 + (e & 1);
                const float v = d[e] * dsilu(F.h1[mt][nt][e]);
                cs1[nt][e & 1] += v;
                const int rloc = warp * 32 + mt * 16 + g + (e >> 1) * 8;
                S.dh1t[col][rloc] = __float2bfloat16_rn(v);
            }
        }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            float a = cs1[nt][e];
#pragma unroll
            for (int q = 4; q < 32; q <<= 1) a += __shfl_xor_sync(MHPC_FULL, a, q);
            if (g == 0) atomicAdd(&S.db1[nt * 8 + t * 2 + e], a);
        }
    __syncthreads();
    // dW2[n][k] = sum_r dH2[r][n] A1[r][k]: warp w owns n in [16w, 16w+16)
    {
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
        for (int kk = 0; kk < kTrainRows / 16; ++kk) {
            unsigned a[4];
            a[0] = ld32(&S.dh2t[warp * 16 + g][kk * 16 + t * 2]);
            a[1] = ld32(&S.dh2t[warp * 16 + g + 8][kk * 16 + t * 2]);
            a[2] = ld32(&S.dh2t[warp * 16 + g][kk * 16 + t * 2 + 8]);
            a[3] = ld32(&S.dh2t[warp * 16 + g + 8][kk * 16 + t * 2 + 8]);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                unsigned b[2];
                b[0] = ld32(&S.a1t[nt * 8 + g][kk * 16 + t * 2]);
                b[1] = ld32(&S.a1t[nt * 8 + g][kk * 16 + t * 2 + 8]);
                mma16816(acc[nt], a, b);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int nrow = warp * 16 + g + (e >> 1) * 8;
                const int kcol = nt * 8 + t * 2 + (e & 1);
                atomicAdd(&grad[MLP_OFF_W2 + nrow * MLP_H + kcol], acc[nt][e]);
            }
    }
    // dW1[n][k] = sum_r dH1[r][n] X[r][k]
    {
        float acc[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
        for (int kk = 0; kk < kTrainRows / 16; ++kk) {
            unsigned a[4];
            a[0] = ld32(&S.dh1t[warp * 16 + g][kk * 16 + t * 2]);
            a[1] = ld32(&S.dh1t[warp * 16 + g + 8][kk * 16 + t * 2]);
            a[2] = ld32(&S.dh1t[warp * 16 + g][kk * 16 + t * 2 + 8]);
            a[3] = ld32(&S.dh1t[warp * 16 + g + 8][kk * 16 + t * 2 + 8]);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                unsigned b[2];
                b[0] = ld32(&S.xt[nt * 8 + g][kk * 16 + t * 2]);
                b[1] = ld32(&S.xt[nt * 8 + g][kk * 16 + t * 2 + 8]);
                mma16816(acc[nt], a, b);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int nrow = warp * 16 + g + (e >> 1) * 8;
                const int kcol = nt * 8 + t * 2 + (e & 1);
                if (kcol < MLP_IN) atomicAdd(&grad[MLP_OFF_W1 + nrow * MLP_INP + kcol], acc[nt][e]);
            }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        atomicAdd(&grad[MLP_OFF_B1 + i], S.db1[i]);
        atomicAdd(&grad[MLP_OFF_B2 + i], S.db2[i]);
        atomicAdd(&grad[MLP_OFF_W3 + i], S.dw3[i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grad[MLP_OFF_B3], S.db3);
        atomicAdd(loss, S.loss);
    }
}

// BF16 copies of the weights in the three layouts the kernels read.
__global__ void k_mirror(const float* __restrict__ w, __nv_bfloat16* w1t, __nv_bfloat16* w2t, __nv_bfloat16* w2k) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_H * MLP_H; i += gridDim.x * blockDim.x) {
        const int nrow = i / MLP_H, k = i % MLP_H;
        const __nv_bfloat16 v = __float2bfloat16_rn(w[MLP_OFF_W2 + i]);
        w2t[i] = v;
        w2k[k * MLP_H + nrow] = v;
        if (i < MLP_H * MLP_INP) w1t[i] = __float2bfloat16_rn(w[MLP_OFF_W1 + i]);
    }
}

__global__ void k_adam(float* w, float* m, float* v, float* grad, float lr, float b1c, float b2c) {
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const float gr = grad[i];
        const float mi = beta1 * m[i] + (1.f - beta1) * gr;
        const float vi = beta2 * v[i] + (1.f - beta2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + eps);
        grad[i] = 0.f;
    }
}

__global__ void k_init_weights(float* w, unsigned long long seed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const unsigned long long r = mix64(seed ^ (0x1234567ULL * (i + 1)));
        const float u = (float)((r >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;  // U(-1, 1)
        float v = 0.f;
        if (i < MLP_OFF_B1) v = (i % MLP_INP) < MLP_IN ? u * sqrtf(3.f / MLP_IN) : 0.f;
        else if (i >= MLP_OFF_W2 && i < MLP_OFF_B2) v = u * sqrtf(3.f / MLP_H);
        else if (i >= MLP_OFF_W3 && i < MLP_OFF_B3) v = u * sqrtf(3.f / MLP_H) * 0.1f;
        w[i] = v;
    }
}

// ------------------------------------------------------- data collection
// Pairs are kept only for particles the plain iteration converged into the
// band (not stopped by the iteration limit) and whose h moved by less than a
// factor 2: the predictor learns the regular evolution of h, not the
// run-away h of particles that cannot reach the band.
__global__ void k_collect(int n, const int* __restrict__ perm, const double* __restrict__ h_start,
                          const double* __restrict__ h_new, const float* __restrict__ feats,
                          const int* __restrict__ count, const int* __restrict__ nit, int target, int tol,
                          int max_iter, int stride, int phase, float* tx, float* ty, unsigned long long* tcount,
                          int tcap) {
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long s = q * stride + phase;
    if (s >= n) return;
    const double hs = h_start[s], hn = h_new[s];
    if (!(hs > 0.0) || !(hn > 0.0)) return;
    if (abs(count[s] - target) >= tol || nit[s] > max_iter || count[s] < 1) return;
    // target: the band-centred h, i.e. the converged h corrected by
    // (target / count)^(1/3) (count ~ h^3), as a log ratio to the starting h
    const double y = log(hn / hs) + log((double)target / (double)count[s]) / 3.0;
    if (fabs(y) >= 0.69) return;
    const int o = perm[s];
    const unsigned long long slot = atomicAdd(tcount, 1ULL) % (unsigned long long)tcap;
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) tx[slot * MLP_IN + k] = feats[(size_t)o * MLP_IN + k];
    ty[slot] = (float)y;
}

__global__ void k_norm_sums(const float* __restrict__ tx, const float* __restrict__ ty,
                            const unsigned long long* tcount, int tcap, double* sums) {
    const unsigned long long cnt = *tcount;
    const long avail = (long)(cnt < (unsigned long long)tcap ? cnt : (unsigned long long)tcap);
    double acc[2 * MLP_IN + 2];
#pragma unroll
    for (int k = 0; k < 2 * MLP_IN + 2; ++k) acc[k] = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < avail; i += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) {
            const double v = tx[i * MLP_IN + k];
            acc[k] += v;
            acc[MLP_IN + k] += v * v;
        }
        const double y = ty[i];
        acc[2 * MLP_IN] += y;
        acc[2 * MLP_IN + 1] += y * y;
    }
#pragma unroll
    for (int k = 0; k < 2 * MLP_IN + 2; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(MHPC_FULL, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sums[k], v);
    }
}

__global__ void k_norm_final(const double* sums, const unsigned long long* tcount, int tcap, float* norm) {
    const unsigned long long cnt = *tcount;
    const double n = (double)(cnt < (unsigned long long)tcap ? cnt : (unsigned long long)tcap);
    if (threadIdx.x < MLP_IN) {
        const int k = threadIdx.x;
        const double mean = n > 0 ? sums[k] / n : 0.0;
        const double var = n > 0 ? fmax(sums[MLP_IN + k] / n - mean * mean, 0.0) : 1.0;
        norm[k] = (float)mean;
        norm[MLP_IN + k] = (float)(1.0 / sqrt(var + 1e-12));
    }
    if (threadIdx.x == 0) {
        const double mean = n > 0 ? sums[2 * MLP_IN] / n : 0.0;
        const double var = n > 0 ? fmax(sums[2 * MLP_IN + 1] / n - mean * mean, 0.0) : 1.0;
        norm[2 * MLP_IN] = (float)mean;
        norm[2 * MLP_IN + 1] = (float)sqrt(var + 1e-12);
    }
}

// --------------------------------------------- features + next-step prediction
constexpr int kFeatBlock = 128;

struct FeatSmem {
    MlpSmem net;
    __nv_bfloat16 xs[kFeatBlock][MLP_INP];
};

__global__ void __launch_bounds__(kFeatBlock) k_features(MlpFeatureInputs in, float* feats, float* hlog,
                                                         double* hbase, const float* __restrict__ w,
                                                         const __nv_bfloat16* w1t, const __nv_bfloat16* w2t,
                                                         const __nv_bfloat16* w2k, const float* norm, int predict) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FeatSmem& S = *reinterpret_cast<FeatSmem*>(smem_raw);
    if (predict) load_net(S.net, w1t, w2t, w2k, w, norm);
    const long s = (long)blockIdx.x * kFeatBlock + threadIdx.x;
    const bool valid = s < in.n;
    const long sl = valid ? s : in.n - 1;
    const int o = in.perm[sl];
    const double h = in.h[sl], rho = in.rho[sl], dt = in.dt;
    const double ax = in.ax[o], ay = in.ay[o], az = in.az[o];
    double g2 = 0.0;
    if (in.gx) g2 = in.gx[o] * in.gx[o] + in.gy[o] * in.gy[o] + in.gz[o] * in.gz[o];
    const double v = sqrt(in.vx[sl] * in.vx[sl] + in.vy[sl] * in.vy[sl] + in.vz[sl] * in.vz[sl]);
    float f[MLP_IN];
    f[0] = (float)log(h);
    f[1] = (float)log(rho);
    f[2] = (float)(-in.drhodt[o] / rho * dt);
    f[3] = (float)((in.noi[sl] - in.target) / (double)in.target);
    f[4] = (float)log(rho * h * h * h / in.m[sl]);
    f[5] = (float)(in.cs[sl] * dt / h);
    f[6] = (float)log(sqrt(ax * ax + ay * ay + az * az) * dt * dt / h + 1e-12);
    f[7] = (float)log(sqrt(g2) * dt * dt / h + 1e-12);
    f[8] = (float)log(h / in.h_start[sl]);
    f[9] = (float)(v * dt / h);
    // (the iteration count is not a feature: it means something else once the
    // iteration starts from predictions)
    f[10] = f[3] * f[3];
    f[11] = (float)log(dt);
    if (valid) {
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) feats[(size_t)o * MLP_IN + k] = f[k];
        hbase[o] = h;
    }
    if (!predict) return;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MLP_INP; ++k) {
        const float x = k < MLP_IN ? (f[k] - S.net.norm[k]) * S.net.norm[MLP_IN + k] : 0.f;
        S.xs[threadIdx.x][k] = __float2bfloat16_rn(x);
    }
    __syncwarp();
    Frags F;
    const float out = warp_forward(S.net, &S.xs[(threadIdx.x >> 5) * 32], F);
    if (valid) hlog[o] = out * S.net.norm[2 * MLP_IN + 1] + S.net.norm[2 * MLP_IN];
}

__global__ void k_apply(int n, const int* __restrict__ perm, const float* __restrict__ hlog,
                        const double* __restrict__ hbase, double* h) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = perm[s];
        const double hb = hbase[o];
        const float l = hlog[o];
        // predictions are clamped to a factor 2 either way of the last h
        if (hb > 0.0 && isfinite(l)) h[s] = hb * exp(fmin(fmax((double)l, -0.69), 0.69));
    }
}

template <typename T>
int dalloc(MlpState* m, T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (count ? count : 1)) != cudaSuccess) return MHPC_ERR_CUDA;
    m->allocs.push_back(q);
    *p = (T*)q;
    return MHPC_OK;
}

size_t train_smem() { return sizeof(TrainSmem); }
size_t feat_smem() { return sizeof(FeatSmem); }

}  // namespace

int mlp_create(MlpState** out, int capacity) {
    MlpState* m = new MlpState();
    m->cap = capacity;
    m->tcap = 1 << 21;
    int rc = MHPC_OK;
#define A(p, c) \
    if (!rc) rc = dalloc(m, &(p), (c))
    A(m->feats, (size_t)capacity * MLP_IN);
    A(m->hlog, capacity);
    A(m->hbase, capacity);
    A(m->w, MLP_NPARAM);
    A(m->adam_m, MLP_NPARAM);
    A(m->adam_v, MLP_NPARAM);
    A(m->grad, MLP_NPARAM);
    A(m->w1t, MLP_H * MLP_INP);
    A(m->w2t, MLP_H * MLP_H);
    A(m->w2k, MLP_H * MLP_H);
    A(m->norm, 2 * MLP_IN + 2);
    A(m->nsum, 2 * MLP_IN + 2);
    A(m->loss, 1);
    A(m->tx, (size_t)m->tcap * MLP_IN);
    A(m->ty, m->tcap);
    A(m->tcount, 1);
#undef A
    if (!rc && cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem()) !=
                   cudaSuccess)
        rc = MHPC_ERR_CUDA;
    if (!rc && cudaFuncSetAttribute(k_features, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)feat_smem()) !=
                   cudaSuccess)
        rc = MHPC_ERR_CUDA;
    if (rc) {
        mlp_destroy(m);
        *out = nullptr;
        return rc;
    }
    *out = m;
    return MHPC_OK;
}

void mlp_destroy(MlpState* m) {
    if (!m) return;
    for (void* p : m->allocs) cudaFree(p);
    delete m;
}

int mlp_ready(const MlpState* m) { return m && m->trained; }
int mlp_has_prediction(const MlpState* m) { return m && m->have_pred; }

int mlp_reset(MlpState* m, unsigned long long seed, cudaStream_t s) {
    k_init_weights<<<32, 256, 0, s>>>(m->w, seed);
    CUDA_TRY(cudaMemsetAsync(m->adam_m, 0, sizeof(float) * MLP_NPARAM, s));
    CUDA_TRY(cudaMemsetAsync(m->adam_v, 0, sizeof(float) * MLP_NPARAM, s));
    CUDA_TRY(cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_NPARAM, s));
    CUDA_TRY(cudaMemsetAsync(m->tcount, 0, sizeof(unsigned long long), s));
    std::vector<float> id(2 * MLP_IN + 2, 0.f);
    for (int k = 0; k < MLP_IN; ++k) id[MLP_IN + k] = 1.f;
    id[2 * MLP_IN + 1] = 1.f;
    CUDA_TRY(cudaMemcpyAsync(m->norm, id.data(), sizeof(float) * id.size(), cudaMemcpyHostToDevice, s));
    k_mirror<<<16, 256, 0, s>>>(m->w, m->w1t, m->w2t, m->w2k);
    CUDA_TRY(cudaStreamSynchronize(s));
    m->adam_t = 0;
    m->trained = 0;
    m->have_pred = 0;
    m->have_feats = 0;
    return cudaGetLastError() == cudaSuccess ? MHPC_OK : MHPC_ERR_CUDA;
}

int mlp_apply_prediction(MlpState* m, const int* perm, double* h_sorted, int n, cudaStream_t s) {
    if (!m->have_pred) return MHPC_OK;
    k_apply<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(n, perm, m->hlog, m->hbase, h_sorted);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int mlp_collect(MlpState* m, const int* perm, const double* h_start, const double* h_new, const int* count,
                const int* nit, int target, int tol, int max_iter, int n, cudaStream_t s) {
    if (!m->have_feats) return MHPC_OK;
    const int stride = n > 65536 ? (n + 65535) / 65536 : 1;
    const int phase = m->step % stride;
    const long cnt = (n - phase + stride - 1) / stride;
    k_collect<<<(int)((cnt + 255) / 256), 256, 0, s>>>(n, perm, h_start, h_new, m->feats, count, nit, target, tol,
                                                       max_iter, stride, phase, m->tx, m->ty, m->tcount, m->tcap);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int mlp_features_predict(MlpState* m, const MlpFeatureInputs& in, cudaStream_t s) {
    const int predict = m->trained;
    const int blocks = (in.n + kFeatBlock - 1) / kFeatBlock;
    k_features<<<blocks, kFeatBlock, feat_smem(), s>>>(in, m->feats, m->hlog, m->hbase, m->w, m->w1t, m->w2t, m->w2k,
                                                       m->norm, predict);
    CUDA_TRY(cudaGetLastError());
    m->have_feats = 1;
    m->have_pred = predict;
    m->step++;
    return MHPC_OK;
}

int mlp_train(MlpState* m, int iters, float lr, int batch, float* loss_out, cudaStream_t s) {
    unsigned long long cnt = 0;
    CUDA_TRY(cudaMemcpyAsync(&cnt, m->tcount, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (cnt < 1024) return MHPC_ERR_ARG;  // not enough (features, h) pairs yet
    if (m->adam_t == 0) {
        CUDA_TRY(cudaMemsetAsync(m->nsum, 0, sizeof(double) * (2 * MLP_IN + 2), s));
        k_norm_sums<<<148, 256, 0, s>>>(m->tx, m->ty, m->tcount, m->tcap, m->nsum);
        k_norm_final<<<1, 32, 0, s>>>(m->nsum, m->tcount, m->tcap, m->norm);
    }
    const int blocks = (batch + kTrainRows - 1) / kTrainRows;
    for (int it = 0; it < iters; ++it) {
        CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(float), s));
        k_train<<<blocks, kTrainRows, train_smem(), s>>>(m->tx, m->ty, batch, m->tcount, m->tcap,
                                                         0x5eed0000ULL + (unsigned long long)m->adam_t * 7919ULL,
                                                         m->w, m->w1t, m->w2t, m->w2k, m->norm, 1, m->grad,
                                                         m->loss, nullptr);
        ++m->adam_t;
        const float b1c = 1.f - powf(0.9f, (float)m->adam_t), b2c = 1.f - powf(0.999f, (float)m->adam_t);
        k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->w, m->adam_m, m->adam_v, m->grad, lr, b1c, b2c);
        k_mirror<<<16, 256, 0, s>>>(m->w, m->w1t, m->w2t, m->w2k);
    }
    CUDA_TRY(cudaGetLastError());
    if (loss_out) {
        CUDA_TRY(cudaMemcpyAsync(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    m->trained = 1;
    return MHPC_OK;
}

int mlp_refresh(MlpState* m, int iters, float lr, int batch, cudaStream_t s) {
    if (!m->trained || iters <= 0) return MHPC_OK;
    const int blocks = (batch + kTrainRows - 1) / kTrainRows;
    for (int it = 0; it < iters; ++it) {
        CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(float), s));
        k_train<<<blocks, kTrainRows, train_smem(), s>>>(m->tx, m->ty, batch, m->tcount, m->tcap,
                                                         0x5eed0000ULL + (unsigned long long)m->adam_t * 7919ULL,
                                                         m->w, m->w1t, m->w2t, m->w2k, m->norm, 1, m->grad,
                                                         m->loss, nullptr);
        ++m->adam_t;
        const float b1c = 1.f - powf(0.9f, (float)m->adam_t), b2c = 1.f - powf(0.999f, (float)m->adam_t);
        k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->w, m->adam_m, m->adam_v, m->grad, lr, b1c, b2c);
        k_mirror<<<16, 256, 0, s>>>(m->w, m->w1t, m->w2t, m->w2k);
    }
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int mlp_forward_backward(MlpState* m, const float* feats, int rows, const float* target, float* out, float* grad,
                         float* loss_out, cudaStream_t s) {
    CUDA_TRY(cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_NPARAM, s));
    CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(float), s));
    const int blocks = (rows + kTrainRows - 1) / kTrainRows;
    k_train<<<blocks, kTrainRows, train_smem(), s>>>(feats, target, rows, nullptr, 0, 0, m->w, m->w1t, m->w2t,
                                                     m->w2k, m->norm, 0, m->grad, m->loss, out);
    CUDA_TRY(cudaGetLastError());
    if (grad) CUDA_TRY(cudaMemcpyAsync(grad, m->grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToDevice, s));
    if (loss_out) CUDA_TRY(cudaMemcpyAsync(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_NPARAM, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return MHPC_OK;
}

int mlp_get_params(MlpState* m, float* host, cudaStream_t s) {
    CUDA_TRY(cudaMemcpyAsync(host, m->w, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return MHPC_OK;
}

int mlp_set_params(MlpState* m, const float* host, cudaStream_t s) {
    CUDA_TRY(cudaMemcpyAsync(m->w, host, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, s));
    k_mirror<<<16, 256, 0, s>>>(m->w, m->w1t, m->w2t, m->w2k);
    CUDA_TRY(cudaStreamSynchronize(s));
    return cudaGetLastError() == cudaSuccess ? MHPC_OK : MHPC_ERR_CUDA;
}
