// Tree construction from sorted keys and the bottom-up moment pass.
//
// Node set: equal, as a set of (key prefix, level), to the reference's
// buildTree result (src/subdomain_key_tree/tree.cu:768-1082); node numbering
// is depth-first pre-order instead of atomic insertion order.  Centres of mass
// follow calculateCentersOfMass (tree.cu:1416-1497): m = sum of child masses,
// x = sum(x_c m_c) / m over the children in curve order, computed with
// explicitly rounded FP64 multiplies and adds (the reference builds with
// -fmad=false) so that Lebesgue-ordered results match it bit for bit.  Like
// the reference (21 launches, miluphpc.cpp:1205-1210) the pass runs one
// launch per level, deepest first, each over a dense list of that level's
// cells built once per tree from the sorted keys' common-digit counts; no
// atomics or fences are involved.
#include "tree.cuh"

namespace {

__device__ __forceinline__ int dl_at(const unsigned char* dl, int i) { return i >= 0 ? (int)dl[i] : 0; }

__global__ void __launch_bounds__(256) k_lcp(const uint64_t* __restrict__ k, int n, unsigned char* dl, int* cnt,
                                             DevStatus* st) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int d = 0;
        if (i + 1 < n) {
            uint64_t x = __ldg(k + i) ^ __ldg(k + i + 1);
            d = x == 0 ? MHPC_MAX_LEVEL : (__clzll((long long)x) - 1) / 3;
            if (d > MHPC_MAX_LEVEL) d = MHPC_MAX_LEVEL;
            if (x == 0) atomicAdd(&st->key_collisions, 1);
        }
        dl[i] = (unsigned char)d;
    }
}

__global__ void __launch_bounds__(256) k_count(const unsigned char* __restrict__ dl, int n, int* cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int dp = dl_at(dl, i - 1), dc = dl[i];
        cnt[i] = (dc > dp ? dc - dp : 0) + 1;
    }
}

// last j in [a, n) whose key shares the prefix (key >> sh) == pref
__device__ int gallop_fwd(const uint64_t* __restrict__ k, int a, int n, uint64_t pref, int sh) {
    int lo = a, hi, step = 1;
    for (;;) {
        long h = (long)lo + step;
        if (h >= n || (__ldg(k + h) >> sh) != pref) { hi = (int)(h < n ? h : n); break; }
        lo = (int)h;
        step <<= 1;
    }
    while (hi - lo > 1) {
        int mid = lo + ((hi - lo) >> 1);
        if ((__ldg(k + mid) >> sh) == pref) lo = mid; else hi = mid;
    }
    return lo;
}

// first j in [0, a] whose key shares the prefix
__device__ int gallop_back(const uint64_t* __restrict__ k, int a, uint64_t pref, int sh) {
    int hi = a, lo, step = 1;
    for (;;) {
        long l = (long)hi - step;
        if (l < 0 || (__ldg(k + l) >> sh) != pref) { lo = (int)(l < 0 ? -1 : l); break; }
        hi = (int)l;
        step <<= 1;
    }
    while (hi - lo > 1) {
        int mid = lo + ((hi - lo) >> 1);
        if ((__ldg(k + mid) >> sh) == pref) hi = mid; else lo = mid;
    }
    return hi;
}

__device__ __forceinline__ int cell_node(const int* off, const unsigned char* dl, int a, int L) {
    return off[a] + (L - dl_at(dl, a - 1) - 1);
}

// Child slot of `node` (level Lc) in its parent: the key digit at level Lc,
// unique among siblings, so slots listed by digit are in curve (pre-)order.
// Leaves below level 21 (particles sharing a full key) have no digit: the
// parent is flagged and its children are then enumerated by skip pointers.
__device__ __forceinline__ void add_kid(TreeDev& T, int par, int node, uint64_t key, int Lc) {
    if (Lc <= MHPC_MAX_LEVEL) {
        const int d = (int)((key >> (3 * (MHPC_MAX_LEVEL - Lc))) & 7);
        T.kids[8 * (size_t)par + d] = node;
        atomicOr(&T.kmask[par], 1 << d);
    } else {
        atomicOr(&T.kmask[par], 0x100);
    }
}

__global__ void __launch_bounds__(256) k_nodes(TreeDev T, const uint64_t* __restrict__ k, DevStatus* st) {
    const int n = T.n;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const int dp = dl_at(T.dl, a - 1), dc = T.dl[a];
        const int c = dc > dp ? dc - dp : 0;
        const int o = T.off[a];
        const uint64_t ka = __ldg(k + a);
        for (int j = 0; j < c; ++j) {
            const int L = dp + 1 + j;
            const int node = o + j;
            if (node >= T.cap_nodes) { set_status(st, MHPC_ERR_NODE_POOL, node); break; }
            const int sh = 3 * (MHPC_MAX_LEVEL - L);
            const int b = gallop_fwd(k, a, n, ka >> sh, sh);
            int par;
            if (j > 0) par = node - 1;
            else if (L - 1 == 0) par = -1;
            else {
                const int sh2 = 3 * (MHPC_MAX_LEVEL - (L - 1));
                const int a2 = gallop_back(k, a, ka >> sh2, sh2);
                par = cell_node(T.off, T.dl, a2, L - 1);
            }
            T.link[node] = make_int2(T.off[b + 1], L);
            T.first[node] = a;
            T.last[node] = b;
            T.parent[node] = par;
            if (par >= T.cap_nodes) set_status(st, MHPC_ERR_NODE_POOL, par);
            else if (par >= 0) add_kid(T, par, node, ka, L);
        }
        const int node = o + c;
        if (node >= T.cap_nodes) { set_status(st, MHPC_ERR_NODE_POOL, node); continue; }
        const int P = dp > dc ? dp : dc;
        int par;
        if (P == 0) par = -1;
        else if (dc > dp) par = node - 1;
        else {
            const int sh2 = 3 * (MHPC_MAX_LEVEL - P);
            const int a2 = gallop_back(k, a, ka >> sh2, sh2);
            par = cell_node(T.off, T.dl, a2, P);
        }
        T.link[node] = make_int2(node + 1, (P + 1) | ND_LEAF);
        T.first[node] = a;
        T.last[node] = a;
        T.parent[node] = par;
        T.leaf_node[a] = node;
        if (par >= T.cap_nodes) set_status(st, MHPC_ERR_NODE_POOL, par);
        else if (par >= 0) add_kid(T, par, node, ka, P + 1);
        if (P + 1 > MHPC_MAX_LEVEL) atomicMax(&st->max_level, P + 1);
    }
}

__global__ void k_zero_cells(TreeDev T) {
    // child masks of cells must be zero before k_nodes sets their bits; cells
    // are the non-leaf nodes, whose ids are unknown before the scan, so clear all.
    int total = *T.nodes;
    if (total > T.cap_nodes) total = T.cap_nodes;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) T.kmask[i] = 0;
}

__global__ void k_copy_total(TreeDev T) { *T.nodes = T.off[T.n]; }

__device__ __forceinline__ float rd(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float ru(double v) { return __double2float_ru(v); }

// Cell lists per level.  The level-L cell starting at sorted position a
// exists iff dl[a-1] < L <= dl[a] (its id is off[a] + L - dl[a-1] - 1);
// k_level_count histograms them per block in shared memory, k_level_offsets
// scans the 21 counts, k_level_fill reserves one range per (block, level) and
// scatters the cell ids.  A block takes a fixed chunk of sorted positions, so
// both passes see the same cells; the order inside a level is irrelevant.
constexpr int kLevelChunk = 2048;

__global__ void __launch_bounds__(256) k_level_count(TreeDev T, const DevStatus* st) {
    if (st->code) return;
    __shared__ int h[32];
    if (threadIdx.x < 32) h[threadIdx.x] = 0;
    __syncthreads();
    const int a0 = blockIdx.x * kLevelChunk;
    const int a1 = min(a0 + kLevelChunk, T.n);
    for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        const int dp = dl_at(T.dl, a - 1), dc = T.dl[a];
        for (int L = dp + 1; L <= dc; ++L) atomicAdd(&h[L], 1);
    }
    __syncthreads();
    if (threadIdx.x >= 1 && threadIdx.x <= MHPC_MAX_LEVEL && h[threadIdx.x])
        atomicAdd(&T.level_off[32 + threadIdx.x], h[threadIdx.x]);
}

__global__ void k_level_offsets(TreeDev T) {
    int acc = 0;
    for (int L = 0; L <= MHPC_MAX_LEVEL + 1; ++L) {
        const int c = (L >= 1 && L <= MHPC_MAX_LEVEL) ? T.level_off[32 + L] : 0;
        T.level_off[L] = acc;
        T.level_off[32 + L] = acc;  // fill cursor of level L
        acc += c;
    }
}

__global__ void __launch_bounds__(256) k_level_fill(TreeDev T, const DevStatus* st) {
    if (st->code) return;
    __shared__ int h[32], base[32];
    if (threadIdx.x < 32) h[threadIdx.x] = 0;
    __syncthreads();
    const int a0 = blockIdx.x * kLevelChunk;
    const int a1 = min(a0 + kLevelChunk, T.n);
    for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        const int dp = dl_at(T.dl, a - 1), dc = T.dl[a];
        for (int L = dp + 1; L <= dc; ++L) atomicAdd(&h[L], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int L = threadIdx.x;
        base[L] = (L >= 1 && L <= MHPC_MAX_LEVEL && h[L]) ? atomicAdd(&T.level_off[32 + L], h[L]) : 0;
        h[L] = 0;
    }
    __syncthreads();
    for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        const int dp = dl_at(T.dl, a - 1), dc = T.dl[a];
        const int o = T.off[a];
        for (int L = dp + 1; L <= dc; ++L) {
            const int i = base[L] + atomicAdd(&h[L], 1);
            if (i < T.cap_nodes) T.level_cells[i] = o + (L - dp - 1);
        }
    }
}

// Children of cell p by key digit: slot d holds a child where bit d of the
// mask is set, so visiting d = 0..7 gives the summation order of the
// reference's calculateCentersOfMass (child slots 0..7); shared-key buckets
// (mask bit 0x100) list theirs by skip pointers.
struct Kids {
    int id[8];
    int mask;
};

__device__ __forceinline__ Kids cell_kids(const TreeDev& T, int p) {
    Kids K;
    K.mask = __ldg(T.kmask + p);
    const int4 k0 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)p));
    const int4 k1 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)p) + 1);
    K.id[0] = k0.x; K.id[1] = k0.y; K.id[2] = k0.z; K.id[3] = k0.w;
    K.id[4] = k1.x; K.id[5] = k1.y; K.id[6] = k1.z; K.id[7] = k1.w;
    return K;
}

// Mixed-path walk record of one node (layout in tree.cuh): FP32 hi/lo split
// of the centre of mass, the geometric opening criterion edge^2/theta (-1 for
// leaves), the quadrupole, the link info with the child mask, and M l^3.
__device__ __forceinline__ void put_wrec(const TreeDev& T, int i, double x, double y, double z, double m, int info,
                                         int mask, float4 q0, float2 q1, double edge0, double inv_theta) {
    const float hx = (float)x, hy = (float)y, hz = (float)z;
    float crit = -1.f, ml3 = 0.f;
    if (!(info & ND_LEAF)) {
        const double e = ldexp(edge0, -(info & 0xff));
        crit = (float)(e * e * inv_theta);
        ml3 = (float)(m * e * e * e);
    }
    float4* w = T.wrec + 4 * (size_t)i;
    w[0] = make_float4(hx, hy, hz, (float)m);
    w[1] = make_float4((float)(x - (double)hx), (float)(y - (double)hy), (float)(z - (double)hz), crit);
    w[2] = q0;
    w[3] = make_float4(q1.x, q1.y, __int_as_float((info & 0x1ff) | (mask << 9)), ml3);
}

// Leaves: centre of mass = the particle; with want_quad (mixed walk) the walk
// record as well (a leaf's quadrupole is zero and never read from quad0/1).
__global__ void __launch_bounds__(256) k_upward_leaves(TreeDev T, const double* __restrict__ sx,
                                                       const double* __restrict__ sy, const double* __restrict__ sz,
                                                       const double* __restrict__ sm, int want_quad,
                                                       int want_box, const long long* __restrict__ ord,
                                                       double inv_theta, const DevStatus* st) {
    if (st->code) return;
    const double edge0 = want_quad ? ord_to_dbl(ord[1]) - ord_to_dbl(ord[0]) : 0.0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < T.n; a += gridDim.x * blockDim.x) {
        const int leaf = T.leaf_node[a];
        const double px = __ldg(sx + a), py = __ldg(sy + a), pz = __ldg(sz + a), pm = __ldg(sm + a);
        T.com[leaf] = make_double4(px, py, pz, pm);
        if (want_box) {
            T.bmin[leaf] = make_float4(rd(px), rd(py), rd(pz), 0.f);
            T.bmax[leaf] = make_float4(ru(px), ru(py), ru(pz), 0.f);
        }
        if (want_quad)
            put_wrec(T, leaf, px, py, pz, pm, __ldg(&T.link[leaf].y), 0, make_float4(0.f, 0.f, 0.f, 0.f),
                     make_float2(0.f, 0.f), edge0, inv_theta);
    }
}

// One level of the upward pass: every cell of level L combines its children,
// which the previous launches (deeper levels, leaves) completed.  Centres of
// mass use explicitly rounded products and sums in slot order, so the result
// is bit-identical to the level-wise sums of the reference.
__global__ void __launch_bounds__(256) k_upward_level(TreeDev T, int L, int want_quad, int want_box,
                                                      const long long* __restrict__ ord, double inv_theta,
                                                      const DevStatus* st) {
    if (st->code) return;
    const double edge0 = want_quad ? ord_to_dbl(ord[1]) - ord_to_dbl(ord[0]) : 0.0;
    const int i0 = T.level_off[L], i1 = min(T.level_off[L + 1], T.cap_nodes);
    for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < i1; i += gridDim.x * blockDim.x) {
        const int p = T.level_cells[i];
        const Kids K = cell_kids(T, p);
        double m = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
        float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
        float4 hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        auto add_com = [&](int c) {
            const double4 cc = ldg_d4(&T.com[c]);
            mx = __dadd_rn(mx, __dmul_rn(cc.x, cc.w));
            my = __dadd_rn(my, __dmul_rn(cc.y, cc.w));
            mz = __dadd_rn(mz, __dmul_rn(cc.z, cc.w));
            m = __dadd_rn(m, cc.w);
            if (want_box) {
                const float4 bl = __ldg(&T.bmin[c]), bh = __ldg(&T.bmax[c]);
                lo.x = fminf(lo.x, bl.x); lo.y = fminf(lo.y, bl.y); lo.z = fminf(lo.z, bl.z);
                hi.x = fmaxf(hi.x, bh.x); hi.y = fmaxf(hi.y, bh.y); hi.z = fmaxf(hi.z, bh.z);
            }
        };
        const int2 lkp = __ldg(&T.link[p]);
        const int end = lkp.x;
        if (K.mask & 0x100) {
            for (int c = p + 1; c < end; c = __ldg(&T.link[c].x)) add_com(c);
        } else {
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((K.mask >> d) & 1) add_com(K.id[d]);
        }
        if (m > 0.0) {
            mx = __ddiv_rn(mx, m);
            my = __ddiv_rn(my, m);
            mz = __ddiv_rn(mz, m);
        }
        T.com[p] = make_double4(mx, my, mz, m);
        if (want_box) {
            T.bmin[p] = lo;
            T.bmax[p] = hi;
        }
        if (want_quad) {
            double q[6] = {0, 0, 0, 0, 0, 0};
            auto add_quad = [&](int c) {
                const double4 cc = ldg_d4(&T.com[c]);
                const double s0 = cc.x - mx, s1 = cc.y - my, s2 = cc.z - mz;
                const double ss = s0 * s0 + s1 * s1 + s2 * s2;
                const double w = cc.w;
                q[0] += w * (3.0 * s0 * s0 - ss);
                q[1] += w * 3.0 * s0 * s1;
                q[2] += w * 3.0 * s0 * s2;
                q[3] += w * (3.0 * s1 * s1 - ss);
                q[4] += w * 3.0 * s1 * s2;
                q[5] += w * (3.0 * s2 * s2 - ss);
                if (!(__ldg(&T.link[c].y) & ND_LEAF)) {
                    const float4 a0 = __ldg(&T.quad0[c]);
                    const float2 a1 = __ldg(&T.quad1[c]);
                    q[0] += a0.x; q[1] += a0.y; q[2] += a0.z; q[3] += a0.w; q[4] += a1.x; q[5] += a1.y;
                }
            };
            if (K.mask & 0x100) {
                for (int c = p + 1; c < end; c = __ldg(&T.link[c].x)) add_quad(c);
            } else {
#pragma unroll
                for (int d = 0; d < 8; ++d)
                    if ((K.mask >> d) & 1) add_quad(K.id[d]);
            }
            const float4 q0 = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
            const float2 q1 = make_float2((float)q[4], (float)q[5]);
            T.quad0[p] = q0;
            T.quad1[p] = q1;
            put_wrec(T, p, mx, my, mz, m, lkp.y, K.mask, q0, q1, edge0, inv_theta);
        }
    }
}

// Bottom-up maximum of the smoothing lengths, level by level like the
// centres of mass.
__global__ void __launch_bounds__(256) k_hmax_leaves(TreeDev T, const double* __restrict__ h, const DevStatus* st) {
    if (st->code) return;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < T.n; a += gridDim.x * blockDim.x)
        T.hmax[T.leaf_node[a]] = __double2float_ru(h[a]);
}

__global__ void __launch_bounds__(256) k_hmax_level(TreeDev T, int L, const DevStatus* st) {
    if (st->code) return;
    const int i0 = T.level_off[L], i1 = min(T.level_off[L + 1], T.cap_nodes);
    for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < i1; i += gridDim.x * blockDim.x) {
        const int p = T.level_cells[i];
        const Kids K = cell_kids(T, p);
        float m = 0.f;
        if (K.mask & 0x100) {
            const int end = __ldg(&T.link[p].x);
            for (int c = p + 1; c < end; c = __ldg(&T.link[c].x)) m = fmaxf(m, __ldg(&T.hmax[c]));
        } else {
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((K.mask >> d) & 1) m = fmaxf(m, __ldg(&T.hmax[K.id[d]]));
        }
        T.hmax[p] = m;
    }
}

}  // namespace

int tree_build(TreeDev& T, const uint64_t* skey, void* scan_scratch, DevStatus* st, cudaStream_t s) {
    const int n = T.n;
    if (n <= 0) return MHPC_ERR_ARG;
    const int g = grid_for(n, 256, 148 * 16);
    k_lcp<<<g, 256, 0, s>>>(skey, n, T.dl, T.cnt, st);
    k_count<<<g, 256, 0, s>>>(T.dl, n, T.cnt);
    CUDA_TRY(cudaGetLastError());
    int rc = scan_exclusive_i32(T.cnt, T.off, n, scan_scratch, s);
    if (rc) return rc;
    k_copy_total<<<1, 1, 0, s>>>(T);
    k_zero_cells<<<148 * 8, 256, 0, s>>>(T);
    k_nodes<<<g, 256, 0, s>>>(T, skey, st);
    CUDA_TRY(cudaMemsetAsync(T.level_off, 0, 64 * sizeof(int), s));
    const int chunks = (n + kLevelChunk - 1) / kLevelChunk;
    k_level_count<<<chunks, 256, 0, s>>>(T, st);
    k_level_offsets<<<1, 1, 0, s>>>(T);
    k_level_fill<<<chunks, 256, 0, s>>>(T, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int tree_upward(TreeDev& T, const double* sx, const double* sy, const double* sz, const double* sm,
                int want_quad, int want_box, const long long* ord, double theta, DevStatus* st, cudaStream_t s) {
    const double inv_theta = want_quad ? 1.0 / theta : 0.0;
    k_upward_leaves<<<grid_for(T.n, 256, 148 * 16), 256, 0, s>>>(T, sx, sy, sz, sm, want_quad, want_box, ord,
                                                                  inv_theta, st);
    const int gl = grid_for(T.n / 2 + 1, 256, 148 * 16);
    for (int L = MHPC_MAX_LEVEL; L >= 1; --L)
        k_upward_level<<<gl, 256, 0, s>>>(T, L, want_quad, want_box, ord, inv_theta, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int tree_node_hmax(const TreeDev& T, const double* h, const DevStatus* st, cudaStream_t s) {
    k_hmax_leaves<<<grid_for(T.n, 256, 148 * 16), 256, 0, s>>>(T, h, st);
    const int gl = grid_for(T.n / 2 + 1, 256, 148 * 16);
    for (int L = MHPC_MAX_LEVEL; L >= 1; --L) k_hmax_level<<<gl, 256, 0, s>>>(T, L, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

