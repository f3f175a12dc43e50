// Tree construction from sorted keys and the bottom-up moment pass.
//
// Node set: equal, as a set of (key prefix, level), to the reference's
// buildTree result (src/subdomain_key_tree/tree.cu:768-1082); node numbering
// is depth-first pre-order instead of atomic insertion order.  Centres of mass
// follow calculateCentersOfMass (tree.cu:1416-1497): m = sum of child masses,
// x = sum(x_c m_c) / m over the children in curve order, computed with
// explicitly rounded FP64 multiplies and adds (the reference builds with
// -fmad=false) so that Lebesgue-ordered results match it bit for bit.  The
// reference runs one launch per level (21 launches, miluphpc.cpp:1205-1210);
// here one launch does the whole pass: each block completes the subtrees
// inside its range of sorted particles level by level between block
// barriers, and the few cells that cross a range boundary by counted
// hand-offs (k_upward below).  The level-L cell starting at sorted position
// a exists iff dl[a-1] < L <= dl[a]; its id is off[a] + L - dl[a-1] - 1.
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
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        T.kmask[i] = 0;
        T.arrive[i] = 0;
    }
}

__global__ void k_copy_total(TreeDev T) { *T.nodes = T.off[T.n]; }

__device__ __forceinline__ float rd(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float ru(double v) { return __double2float_ru(v); }

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

// Loads of values that the running upward pass itself writes, never through
// the non-coherent read-only path: written by this block (`local`), cached
// in L1, which sees the block's own stores; written by another block,
// through L2 (ld.global.cg).
template <typename V>
__device__ __forceinline__ V ld_up(const V* p, bool local) {
    return local ? *p : __ldcg(p);
}
__device__ __forceinline__ double4 ld_up_d4(const double4* p, bool local) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = ld_up(q, local), b = ld_up(q + 1, local);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Leaf: centre of mass = the particle; with want_quad (mixed walk) the walk
// record as well (a leaf's quadrupole is zero; its record's leaf flag says so).
__device__ __forceinline__ void leaf_moments(const TreeDev& T, int a, int leaf, const double* __restrict__ sx,
                                             const double* __restrict__ sy, const double* __restrict__ sz,
                                             const double* __restrict__ sm, int want_quad, int want_box,
                                             double edge0, double inv_theta) {
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

// Cell p from its completed children.  Centres of mass use explicitly
// rounded products and sums in slot order, so the result is bit-identical to
// the level-wise sums of the reference.  With `local` the first pass over the
// children also brings their quadrupoles into L1 for the second.
__device__ __forceinline__ void cell_moments(const TreeDev& T, int p, const Kids& K, int want_quad, int want_box,
                                             double edge0, double inv_theta, bool local) {
    double m = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    float4 hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    auto add_com = [&](int c) {
        const double4 cc = ld_up_d4(&T.com[c], local);
        if (local && want_quad) prefetch_l1(T.wrec + 4 * (size_t)c + 2);
        mx = __dadd_rn(mx, __dmul_rn(cc.x, cc.w));
        my = __dadd_rn(my, __dmul_rn(cc.y, cc.w));
        mz = __dadd_rn(mz, __dmul_rn(cc.z, cc.w));
        m = __dadd_rn(m, cc.w);
        if (want_box) {
            const float4 bl = ld_up(&T.bmin[c], local), bh = ld_up(&T.bmax[c], local);
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
            const double4 cc = ld_up_d4(&T.com[c], local);
            const double s0 = cc.x - mx, s1 = cc.y - my, s2 = cc.z - mz;
            const double ss = s0 * s0 + s1 * s1 + s2 * s2;
            const double w = cc.w;
            q[0] += w * (3.0 * s0 * s0 - ss);
            q[1] += w * 3.0 * s0 * s1;
            q[2] += w * 3.0 * s0 * s2;
            q[3] += w * (3.0 * s1 * s1 - ss);
            q[4] += w * 3.0 * s1 * s2;
            q[5] += w * (3.0 * s2 * s2 - ss);
            // the child's quadrupole from its walk record (one 32-byte sector)
            const float4 a0 = ld_up(T.wrec + 4 * (size_t)c + 2, local);
            const float4 a1 = ld_up(T.wrec + 4 * (size_t)c + 3, local);
            if (!(__float_as_int(a1.z) & ND_LEAF)) {
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
        put_wrec(T, p, mx, my, mz, m, lkp.y, K.mask, q0, q1, edge0, inv_theta);
    }
}

// The upward pass in one launch.  Block b owns the sorted particles
// [a0, a1) = [b C, (b + 1) C): it completes their leaves, then, deepest level
// first with a block barrier between levels, every cell that starts and ends
// inside the range (cells starting at position a are levels dl[a-1]+1 ..
// dl[a]); their children are its own leaves and cells, so no other block is
// involved and their loads go through L1, which holds the block's own
// stores.  Whether a cell ends inside the range, and whether a parent crosses
// a range boundary, follows from the block's prefix and suffix minima of dl
// in shared memory, without a load.  Each warp queues its cells of the level
// in shared memory and spreads them over its lanes, so a level costs one
// combine per lane, not one per owned position.  A cell that crosses a range
// boundary collects its
// children by a count instead: the block's completed nodes whose parent
// crosses are queued and handed off after the last level (every thread
// fences its own writes, then one barrier), and each hand-off adds one to the
// parent's count; the thread that adds the last combines the parent and
// hands it off in turn (fence, count, fence, combine).  The combining thread
// clears the count for the next pass over the same tree.  Crossing cells are
// the common ancestors of the two particles at a range boundary, at most 21
// per boundary, so counted hand-offs are rare.
// 256 threads x 8 positions; 4 resident blocks per SM (64 registers) measured
// faster than 2 (86 registers); 16 positions per thread measured slower
constexpr int kUpBlock = 256;
constexpr int kUpPer = 8;  // positions per thread
constexpr int kUpChunk = kUpPer * kUpBlock;
constexpr int kUpHand = 1024;

__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// children of cell p: digit slots, or for a shared-key bucket its particles (all leaves)
__device__ __forceinline__ int cell_nkids(const TreeDev& T, int p) {
    const int mask = __ldg(T.kmask + p);
    return (mask & 0x100) ? __ldg(T.last + p) - __ldg(T.first + p) + 1 : __popc(mask & 0xff);
}

// one completed child of p counted (after the caller's release fence)
template <typename Combine>
__device__ __forceinline__ void hand_off(const TreeDev& T, int p, Combine&& combine) {
    while (p >= 0) {
        const int need = cell_nkids(T, p);
        if (atomicAdd(T.arrive + p, 1) != need - 1) return;
        fence_acq_rel();
        T.arrive[p] = 0;
        combine(p, false);
        fence_acq_rel();
        p = __ldg(T.parent + p);
    }
}

// Minimum over the block of per-thread aggregates, exclusive, from the left
// (prefix) or from the right (suffix); identity 255.
__device__ __forceinline__ void block_min_scans(int agg, int* wtot, int& pre, int& suf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int p = agg, q = agg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(MHPC_FULL, p, o);
        const int w = __shfl_down_sync(MHPC_FULL, q, o);
        if (lane >= o) p = min(p, v);
        if (lane + o < 32) q = min(q, w);
    }
    // p, q: inclusive within the warp; totals per warp to shared memory
    if (lane == 31) wtot[warp] = p;
    __syncthreads();
    int left = 255, right = 255;
    for (int w = 0; w < kUpBlock / 32; ++w) {
        if (w < warp) left = min(left, wtot[w]);
        if (w > warp) right = min(right, wtot[w]);
    }
    const int pe = __shfl_up_sync(MHPC_FULL, p, 1), qe = __shfl_down_sync(MHPC_FULL, q, 1);
    pre = min(left, lane > 0 ? pe : 255);
    suf = min(right, lane < 31 ? qe : 255);
}

template <typename Leaf, typename Combine>
__device__ __forceinline__ void upward_chunk(const TreeDev& T, Leaf&& leaf_fn, Combine&& combine) {
    __shared__ int queue[kUpBlock / 32][32 * kUpPer];             // cell
    __shared__ unsigned short qpos[kUpBlock / 32][32 * kUpPer];   // its first position - a0
    __shared__ int hand[kUpHand];
    // dls[i + 1] = dl[a0 + i], dls[0] = dl[a0 - 1]; pre[i] = min dl[a0 - 1 .. a - 1],
    // suf[i] = min dl[a .. a1 - 1] for a = a0 + i: the run of common digits >= L
    // through position a leaves the range to the left iff pre[i] >= L, to the
    // right iff suf[i] >= L
    __shared__ unsigned char dls[kUpChunk + 1], pre[kUpChunk], suf[kUpChunk];
    __shared__ int wtot[kUpBlock / 32];
    __shared__ int nhand, smax;
    const int a0 = blockIdx.x * kUpChunk, a1 = min(a0 + kUpChunk, T.n), na = a1 - a0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) { nhand = 0; smax = 0; dls[0] = (unsigned char)dl_at(T.dl, a0 - 1); }
    {
        // thread t: positions kUpPer t .. kUpPer t + kUpPer - 1
        int v[kUpPer], agg = 255, mx = 0;
#pragma unroll
        for (int k = 0; k < kUpPer; ++k) {
            const int i = kUpPer * threadIdx.x + k;
            v[k] = i < na ? (int)T.dl[a0 + i] : 255;
            agg = min(agg, v[k]);
            if (i < na) mx = max(mx, v[k]);
        }
        int el, er;
        block_min_scans(agg, wtot, el, er);  // (contains a barrier: nhand, smax, dls[0] are set)
        el = min(el, (int)dls[0]);
        int run = el;
#pragma unroll
        for (int k = 0; k < kUpPer; ++k) {
            const int i = kUpPer * threadIdx.x + k;
            if (i < na) { pre[i] = (unsigned char)run; dls[i + 1] = (unsigned char)v[k]; }
            run = min(run, v[k]);
        }
        run = er;
#pragma unroll
        for (int k = kUpPer - 1; k >= 0; --k) {
            const int i = kUpPer * threadIdx.x + k;
            run = min(run, v[k]);
            if (i < na) suf[i] = (unsigned char)run;
        }
        mx = __reduce_max_sync(MHPC_FULL, mx);
        if (lane == 0) atomicMax(&smax, mx);
    }
    __syncthreads();
    auto queue_parent = [&](int node) {
        const int p = __ldg(T.parent + node);
        const int i = atomicAdd(&nhand, 1);
        if (i < kUpHand) {
            hand[i] = p;
        } else {  // queue full (not reached for kUpChunk particles): hand off at once
            fence_acq_rel();
            hand_off(T, p, combine);
        }
    };
#pragma unroll 2
    for (int j = 0; j < kUpPer; ++j) {
        const int i = j * kUpBlock + threadIdx.x;
        if (i >= na) break;
        const int leaf = T.leaf_node[a0 + i];
        leaf_fn(a0 + i, leaf);
        // parent: the cell of level P = max(dl[a-1], dl[a]) (none for P = 0)
        const int P = max((int)dls[i], (int)dls[i + 1]);
        if (P > 0 && (pre[i] >= P || suf[i] >= P)) queue_parent(leaf);
    }
    int* q = queue[warp];
    unsigned short* qi = qpos[warp];
    for (int L = MHPC_MAX_LEVEL; L >= 1; --L) {
        __syncthreads();
        if (L > smax) continue;  // uniform
        // this lane's local cells of level L (start in the range, end inside it), queued for the warp
        unsigned sel = 0;
#pragma unroll
        for (int j = 0; j < kUpPer; ++j) {
            const int i = j * kUpBlock + threadIdx.x;
            if (i < na && dls[i] < L && L <= dls[i + 1] && suf[i] < L) sel |= 1u << j;
        }
        const int c = __popc(sel);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(MHPC_FULL, incl, 31);
        int w = incl - c;
        while (sel) {
            const int j = __ffs(sel) - 1;
            sel &= sel - 1;
            const int i = j * kUpBlock + threadIdx.x;
            q[w] = T.off[a0 + i] + (L - dls[i] - 1);
            qi[w++] = (unsigned short)i;
        }
        __syncwarp();
        for (int k = lane; k < total; k += 32) {
            const int p = q[k];
            combine(p, true);
            // parent of level L - 1 crossing a range boundary: queued for the hand-off
            const int i = qi[k];
            if (L > 1 && (pre[i] >= L - 1 || suf[i] >= L - 1)) queue_parent(p);
        }
        __syncwarp();
    }
    // hand-offs: every thread releases its own writes, then the queued parents are counted
    fence_acq_rel();
    __syncthreads();
    const int nh = min(nhand, kUpHand);
    for (int k = threadIdx.x; k < nh; k += kUpBlock) hand_off(T, hand[k], combine);
}

__global__ void __launch_bounds__(kUpBlock, 4) k_upward(TreeDev T, const double* __restrict__ sx,
                                                     const double* __restrict__ sy, const double* __restrict__ sz,
                                                     const double* __restrict__ sm, int want_quad, int want_box,
                                                     const long long* __restrict__ ord, double inv_theta,
                                                     const DevStatus* st) {
    if (st->code) return;
    const double edge0 = want_quad ? ord_to_dbl(ord[1]) - ord_to_dbl(ord[0]) : 0.0;
    upward_chunk(
        T, [&](int a, int leaf) { leaf_moments(T, a, leaf, sx, sy, sz, sm, want_quad, want_box, edge0, inv_theta); },
        [&](int p, bool local) {
            cell_moments(T, p, cell_kids(T, p), want_quad, want_box, edge0, inv_theta, local);
        });
}


// Bottom-up maximum of the smoothing lengths, in one launch like the moments.
__global__ void __launch_bounds__(kUpBlock, 4) k_hmax(TreeDev T, const double* __restrict__ h, const DevStatus* st) {
    if (st->code) return;
    upward_chunk(
        T, [&](int a, int leaf) { T.hmax[leaf] = __double2float_ru(h[a]); },
        [&](int p, bool local) {
            const int km = __ldg(T.kmask + p);
            float m = 0.f;
            if (km & 0x100) {
                const int end = __ldg(&T.link[p].x);
                for (int c = p + 1; c < end; c = __ldg(&T.link[c].x)) m = fmaxf(m, ld_up(&T.hmax[c], local));
            } else {
                const Kids K = cell_kids(T, p);
#pragma unroll
                for (int d = 0; d < 8; ++d)
                    if ((K.mask >> d) & 1) m = fmaxf(m, ld_up(&T.hmax[K.id[d]], local));
            }
            T.hmax[p] = m;
        });
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
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int tree_upward(TreeDev& T, const double* sx, const double* sy, const double* sz, const double* sm,
                int want_quad, int want_box, const long long* ord, double theta, DevStatus* st, cudaStream_t s) {
    const double inv_theta = want_quad ? 1.0 / theta : 0.0;
    k_upward<<<(T.n + kUpChunk - 1) / kUpChunk, kUpBlock, 0, s>>>(T, sx, sy, sz, sm, want_quad, want_box, ord,
                                                                  inv_theta, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int tree_node_hmax(const TreeDev& T, const double* h, const DevStatus* st, cudaStream_t s) {
    k_hmax<<<(T.n + kUpChunk - 1) / kUpChunk, kUpBlock, 0, s>>>(T, h, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

