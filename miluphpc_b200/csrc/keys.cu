// Bounding box and space-filling-curve keys.
//
// computeBoundingBox (src/subdomain_key_tree/tree.cu:302-437) reduced the box
// in 4 blocks behind a mutex; here every block reduces its share and merges
// with two 64-bit atomicMin/atomicMax on an order-preserving integer image of
// the doubles, so one launch covers any n.  The merged box starts at 0, like
// resetArrays (src/device_rhs.cu:24-33), and is cubic (CUBIC_DOMAINS), so a
// single (min, max) pair describes all three axes.
//
// Keys follow Tree::getParticleKey (tree.cu:157-240) bit for bit: 21 levels
// of FP64 midpoint bisection, octant bit set when the coordinate is BELOW the
// midpoint, level l at bits 3*(20-l).  Hilbert keys use the reference's
// DirTable/HilbertTable state machine (tree.cuh:66-79, 120-131; tree.cu:40-53).
#include "common.cuh"

namespace {

__global__ void __launch_bounds__(256) k_bbox(const double* __restrict__ x, const double* __restrict__ y,
                                              const double* __restrict__ z, int n, long long* ord,
                                              DevStatus* st) {
    // st may be null (stateless entry point): non-finite input is then not reported
    double mn = 0.0, mx = 0.0;
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a = __ldg(x + i), b = __ldg(y + i), c = __ldg(z + i);
        bad |= !(isfinite(a) && isfinite(b) && isfinite(c));
        mn = fmin(mn, fmin(a, fmin(b, c)));
        mx = fmax(mx, fmax(a, fmax(b, c)));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(MHPC_FULL, mn, o));
        mx = fmax(mx, __shfl_xor_sync(MHPC_FULL, mx, o));
    }
    __shared__ double smn[8], smx[8];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { smn[w] = mn; smx[w] = mx; }
    if (__any_sync(MHPC_FULL, bad) && l == 0 && st) set_status(st, MHPC_ERR_NAN, -1);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { mn = fmin(mn, smn[k]); mx = fmax(mx, smx[k]); }
        atomicMin(ord + 0, dbl_to_ord(mn));
        atomicMax(ord + 1, dbl_to_ord(mx));
    }
}

__global__ void k_bbox_finish(const long long* ord, double* bb) {
    double mn = ord_to_dbl(ord[0]), mx = ord_to_dbl(ord[1]);
    bb[0] = bb[2] = bb[4] = mn;
    bb[1] = bb[3] = bb[5] = mx;
}

__constant__ unsigned char c_dir[12][8] = {
    {8, 10, 3, 3, 4, 5, 4, 5},  {2, 2, 11, 9, 4, 5, 4, 5},  {7, 6, 7, 6, 8, 10, 1, 1},
    {7, 6, 7, 6, 0, 0, 11, 9},  {0, 8, 1, 11, 6, 8, 6, 11}, {10, 0, 9, 1, 10, 7, 9, 7},
    {10, 4, 9, 4, 10, 2, 9, 3}, {5, 8, 5, 11, 2, 8, 3, 11}, {4, 9, 0, 0, 7, 9, 2, 2},
    {1, 1, 8, 5, 3, 3, 8, 6},   {11, 5, 0, 0, 11, 6, 2, 2}, {1, 1, 4, 10, 3, 3, 7, 10}};
__constant__ unsigned char c_hil[12][8] = {
    {0, 7, 3, 4, 1, 6, 2, 5}, {4, 3, 7, 0, 5, 2, 6, 1}, {6, 1, 5, 2, 7, 0, 4, 3},
    {2, 5, 1, 6, 3, 4, 0, 7}, {0, 1, 7, 6, 3, 2, 4, 5}, {6, 7, 1, 0, 5, 4, 2, 3},
    {2, 3, 5, 4, 1, 0, 6, 7}, {4, 5, 3, 2, 7, 6, 0, 1}, {0, 3, 1, 2, 7, 4, 6, 5},
    {2, 1, 3, 0, 5, 6, 4, 7}, {4, 7, 5, 6, 3, 0, 2, 1}, {6, 5, 7, 4, 1, 2, 0, 3}};

// Midpoint bisection of one coordinate for 21 levels; returns the 21 octant
// bits of this axis, bit (20 - level) set when the coordinate is below the
// midpoint.  The midpoints are formed exactly as 0.5 * (min + max) in FP64.
__device__ __forceinline__ uint32_t axis_bits(double v, double lo, double hi) {
    uint32_t bits = 0;
#pragma unroll
    for (int level = 0; level < 21; ++level) {
        double mid = __dmul_rn(0.5, __dadd_rn(lo, hi));
        bool below = v < mid;
        bits = (bits << 1) | (below ? 1u : 0u);
        hi = below ? mid : hi;
        lo = below ? lo : mid;
    }
    return bits;
}

// Interleave: axis bit b of level l goes to key bit 3*(20-l) + axis.
__device__ __forceinline__ uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffffULL;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

__global__ void __launch_bounds__(256) k_keys(const double* __restrict__ x, const double* __restrict__ y,
                                              const double* __restrict__ z, int n,
                                              const long long* __restrict__ ord, const double* __restrict__ bb,
                                              int curve, uint64_t* __restrict__ keys, int* __restrict__ iota) {
    // two levels per lookup: state s and the octants (c1, c2) of two
    // consecutive levels -> (Hilbert digits h1 h2 as 6 bits) | (state after both) << 6,
    // composed from the one-level tables, so the result is the same
    __shared__ unsigned short s2[12 * 64];
    if (curve == 1) {
        for (int e = threadIdx.x; e < 12 * 64; e += blockDim.x) {
            const int st = e >> 6, c1 = (e >> 3) & 7, c2 = e & 7;
            const int h1 = c_hil[st][c1], st1 = c_dir[st][c1];
            const int h2 = c_hil[st1][c2], st2 = c_dir[st1][c2];
            s2[e] = (unsigned short)((h1 << 3) | h2 | (st2 << 6));
        }
    }
    __syncthreads();
    const double lo = bb ? bb[0] : ord_to_dbl(ord[0]), hi = bb ? bb[1] : ord_to_dbl(ord[1]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t bx = axis_bits(__ldg(x + i), lo, hi);
        uint32_t by = axis_bits(__ldg(y + i), lo, hi);
        uint32_t bz = axis_bits(__ldg(z + i), lo, hi);
        uint64_t key = spread3(bx) | (spread3(by) << 1) | (spread3(bz) << 2);
        if (curve == 1) {
            // levels 21..2 in pairs, then level 1
            uint64_t h = 0;
            int dir = 0;
#pragma unroll
            for (int lvl = 21; lvl > 1; lvl -= 2) {
                const int e = s2[(dir << 6) | (int)((key >> (3 * (lvl - 2))) & 63ULL)];
                h = (h << 6) | (uint64_t)(e & 63);
                dir = e >> 6;
            }
            const int e = s2[(dir << 6) | (int)((key & 7ULL) << 3)];  // (c1, c2 = 0): h1 in bits 3-5
            key = (h << 3) | (uint64_t)((e >> 3) & 7);
        }
        keys[i] = key;
        if (iota) iota[i] = i;
    }
}

}  // namespace

int launch_bbox(const double* x, const double* y, const double* z, int n, long long* ord,
                DevStatus* st, cudaStream_t s) {
    CUDA_TRY(cudaMemsetAsync(ord, 0, 2 * sizeof(long long), s));
    if (n > 0) {
        k_bbox<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(x, y, z, n, ord, st);
        CUDA_TRY(cudaGetLastError());
    }
    return MHPC_OK;
}

int launch_bbox_finish(const long long* ord, double* bb, cudaStream_t s) {
    k_bbox_finish<<<1, 1, 0, s>>>(ord, bb);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_keys(const double* x, const double* y, const double* z, int n, const long long* ord,
                int curve, uint64_t* keys, int* iota, cudaStream_t s) {
    if (n <= 0) return MHPC_OK;
    k_keys<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(x, y, z, n, ord, nullptr, curve, keys, iota);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_keys_box(const double* x, const double* y, const double* z, int n, const double* bbox, int curve,
                    uint64_t* keys, cudaStream_t s) {
    if (n <= 0) return MHPC_OK;
    k_keys<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(x, y, z, n, nullptr, bbox, curve, keys, nullptr);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
