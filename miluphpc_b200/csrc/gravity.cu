// Barnes-Hut gravity walks.
//
// Both walks give one warp to 32 consecutive particles of the sorted order,
// exactly the grouping of the reference's computeForces_v2
// (src/gravity/gravity.cu:726-903, launched 256x256 with warps taking
// consecutive `sorted` entries).  The tree is in depth-first pre-order with a
// skip pointer per node, so the walk needs no stack: accepting a node jumps
// to its skip pointer, opening it steps to node+1.
#include "gravity.cuh"

namespace {

constexpr int kWalkBlock = 128;
#ifndef MHPC_MIXED_PPL
#define MHPC_MIXED_PPL 2
#endif

// --------------------------------------------------------------- plain v2
// computeForces_v2 semantics: a child is accepted if it is a leaf or if every
// lane has dp(level) <= r, r = |d|^2 + eps2 (warp vote, __all_sync); root
// children (level 1) are always opened; a root child that is a single leaf is
// pushed as a node by the reference and contributes nothing, which is kept.
// r is formed with explicitly rounded products and sums like the
// reference's -fmad=false build so that accept decisions match it exactly.
__global__ void __launch_bounds__(kWalkBlock) k_grav_v2(const double4* __restrict__ com, const int2* __restrict__ link,
                                                        const int* __restrict__ nodes_total, GravParams P,
                                                        const double* __restrict__ sx, const double* __restrict__ sy,
                                                        const double* __restrict__ sz, const double* __restrict__ sh,
                                                        const int* __restrict__ perm, double* __restrict__ gax,
                                                        double* __restrict__ gay, double* __restrict__ gaz,
                                                        DevStatus* st) {
    if (st->code) return;
    const int M = *nodes_total;
    const int lane = threadIdx.x & 31;
    const long gwarp = ((long)blockIdx.x * kWalkBlock + threadIdx.x) >> 5;
    const long ngroups = ((long)P.n + 31) >> 5;
    if (gwarp >= ngroups) return;
    const long s = gwarp * 32 + lane;
    const bool valid = s < P.n;
    double px = 0, py = 0, pz = 0, e2 = P.eps2;
    if (valid) {
        px = __ldg(sx + s); py = __ldg(sy + s); pz = __ldg(sz + s);
        if (P.h_factor > 0.0) { double e = P.h_factor * __ldg(sh + s); e2 += e * e; }
    }
    // dp(L) = (radius^2 / theta) * 0.25^(L-1); powers of two scale exactly,
    // so this equals the reference's repeated 0.25 * depth products.
    const double radius = 0.5 * (ord_to_dbl(P.ord[1]) - ord_to_dbl(P.ord[0]));
    const double depth1 = radius * radius / P.theta;
    double ax = 0, ay = 0, az = 0;
    unsigned long long ninter = 0, nvisit = 0;
    int nd = 0;
    while (nd < M) {
        const int2 lk = __ldg(link + nd);
        const int L = lk.y & 0xff;
        const bool leaf = lk.y & ND_LEAF;
        ++nvisit;
        if (L == 1) {  // root child
            nd = leaf ? lk.x : nd + 1;
            continue;
        }
        const double4 c = ldg_d4(com + nd);
        const double dx = c.x - px, dy = c.y - py, dz = c.z - pz;
        double r = __dadd_rn(__dmul_rn(dx, dx), e2);
        r = __dadd_rn(r, __dmul_rn(dy, dy));
        r = __dadd_rn(r, __dmul_rn(dz, dz));
        bool acc = leaf;
        if (!leaf) acc = __all_sync(MHPC_FULL, !valid || ldexp(depth1, -2 * (L - 1)) <= r);
        if (acc) {
            double f = 0.0;
            if (r > 0.0) {
                const double ri = rsqrt(r);
                f = c.w * ri * ri * ri;
            }
            ax += f * dx; ay += f * dy; az += f * dz;
            ++ninter;
            nd = lk.x;
        } else {
            ++nd;
        }
    }
    if (valid) {
        const int o = __ldg(perm + s);
        gax[o] = P.G * ax; gay[o] = P.G * ay; gaz[o] = P.G * az;
    }
    // statistics: accepted interactions (lanes x nodes) and node visits per warp
    unsigned nv = __popc(__ballot_sync(MHPC_FULL, valid));
    if (lane == 0) {
        atomicAdd(&st->interactions, ninter * nv);
        atomicAdd(&st->nodes_visited, nvisit);
    }
}

// computeForces_v1 semantics (src/gravity/gravity.cu:252-396, gravityForceVersion
// 2): every particle walks the tree on its own (one thread per particle,
// stackless over the pre-order and skip links; the reference keeps a stack of
// child slots, which visits the nodes in the same order for Lebesgue keys).
// A node other than the particle's own leaf is accepted when it is a leaf or
// d^2 theta^2 > cellSize(level), cellSize(1) = radius^2, quartered per level;
// accepted nodes add m d / |d|^3 with |d| = sqrt(d^2), d^2 formed as dx^2 +
// eps2 + dy^2 + dz^2 in that order, all products and sums explicitly rounded
// like the reference's -fmad=false build.
__global__ void __launch_bounds__(kWalkBlock) k_grav_v1(const double4* __restrict__ com, const int2* __restrict__ link,
                                                        const int* __restrict__ nodes_total,
                                                        const int* __restrict__ leaf_node, GravParams P,
                                                        const double* __restrict__ sh, const int* __restrict__ perm,
                                                        double* __restrict__ gax, double* __restrict__ gay,
                                                        double* __restrict__ gaz, DevStatus* st) {
    if (st->code) return;
    const int M = *nodes_total;
    const long s = (long)blockIdx.x * kWalkBlock + threadIdx.x;
    const bool valid = s < P.n;
    unsigned long long ninter = 0, nvisit = 0;
    if (valid) {
        const int self = __ldg(leaf_node + s);
        const double4 pc = ldg_d4(com + self);
        double e2 = P.eps2;
        if (P.h_factor > 0.0) { const double e = P.h_factor * __ldg(sh + s); e2 += e * e; }
        const double radius = 0.5 * (ord_to_dbl(P.ord[1]) - ord_to_dbl(P.ord[0]));
        const double cs1 = radius * radius, th2 = P.theta * P.theta;
        double ax = 0, ay = 0, az = 0;
        int nd = 0;
        while (nd < M) {
            const int2 lk = __ldg(link + nd);
            ++nvisit;
            if (nd == self) { nd = lk.x; continue; }
            const double4 c = ldg_d4(com + nd);
            const double dx = c.x - pc.x, dy = c.y - pc.y, dz = c.z - pc.z;
            double d = __dadd_rn(__dmul_rn(dx, dx), e2);
            d = __dadd_rn(d, __dmul_rn(dy, dy));
            d = __dadd_rn(d, __dmul_rn(dz, dz));
            const bool leaf = lk.y & ND_LEAF;
            if (leaf || __dmul_rn(d, th2) > ldexp(cs1, -2 * ((lk.y & 0xff) - 1))) {
                const double r = __dsqrt_rn(d);
                const double f = __ddiv_rn(c.w, __dmul_rn(__dmul_rn(r, r), r));
                ax = __dadd_rn(ax, __dmul_rn(f, dx));
                ay = __dadd_rn(ay, __dmul_rn(f, dy));
                az = __dadd_rn(az, __dmul_rn(f, dz));
                ++ninter;
                nd = lk.x;
            } else {
                ++nd;
            }
        }
        const int o = __ldg(perm + s);
        gax[o] = P.G * ax; gay[o] = P.G * ay; gaz[o] = P.G * az;
    }
    // statistics, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        ninter += __shfl_xor_sync(MHPC_FULL, ninter, o);
        nvisit += __shfl_xor_sync(MHPC_FULL, nvisit, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st->interactions, ninter);
        atomicAdd(&st->nodes_visited, nvisit);
    }
}

// -------------------------------------------------------------- mixed FP32
// The group's centre c (FP64, centre of its bounding box) is subtracted once;
// lanes hold their position relative to c in FP32, nodes are stored as
// float hi + float lo of the FP64 centre of mass, so node - c is formed as
// (hi - c_hi) + (lo - c_lo) without losing the digits that FP32 absolute
// coordinates would drop.  A cell is accepted for the warp when every lane
// has edge^2/theta <= |node - p|^2 (the squared-ratio criterion with
// computeForces_v2's warp vote, applied at every level); accepted cells add
// monopole + quadrupole terms.  A box test per group would be cheaper per
// node but opens the whole interior of a group box that straddles a curve
// jump (Lebesgue order), which leaves single warps with tens of thousands of
// leaf interactions; the per-lane vote keeps the cost of such a group at the
// union of its parts.  FP32 partial sums are flushed into FP64 every kFlush
// accepted nodes (compensated accumulation).
constexpr int kFlush = 64;

// PPL particles per lane: a warp takes 32 * PPL consecutive sorted particles;
// each visited node is loaded, placed in the warp frame and voted on once for
// all of them, which amortises the per-node instructions over PPL
// interactions (the kernel is issue-bound, not memory-bound).
template <int PPL>
__global__ void __launch_bounds__(kWalkBlock) k_grav_mixed(const float4* __restrict__ wrec,
                                                           const int2* __restrict__ link, const int* __restrict__ nodes_total,
                                                           const int* __restrict__ leaf_node,
                                                           GravParams P, const double* __restrict__ sx,
                                                           const double* __restrict__ sy, const double* __restrict__ sz,
                                                           const double* __restrict__ sh, const int* __restrict__ perm,
                                                           double* __restrict__ gax, double* __restrict__ gay,
                                                           double* __restrict__ gaz, DevStatus* st) {
    if (st->code) return;
    const int M = *nodes_total;
    const int lane = threadIdx.x & 31;
    const long gwarp = ((long)blockIdx.x * kWalkBlock + threadIdx.x) >> 5;
    const long ngroups = ((long)P.n + 32 * PPL - 1) / (32 * PPL);
    if (gwarp >= ngroups) return;
    const long s0 = gwarp * 32 * PPL;
    long s[PPL];
    bool valid[PPL];
    double px[PPL], py[PPL], pz[PPL], e2d[PPL];
    double lox = 1e300, loy = 1e300, loz = 1e300, hix = -1e300, hiy = -1e300, hiz = -1e300;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        s[k] = s0 + k * 32 + lane;
        valid[k] = s[k] < P.n;
        const long sl = valid[k] ? s[k] : (long)P.n - 1;
        px[k] = __ldg(sx + sl); py[k] = __ldg(sy + sl); pz[k] = __ldg(sz + sl);
        e2d[k] = P.eps2;
        if (P.h_factor > 0.0) { const double e = P.h_factor * __ldg(sh + sl); e2d[k] += e * e; }
        lox = fmin(lox, px[k]); loy = fmin(loy, py[k]); loz = fmin(loz, pz[k]);
        hix = fmax(hix, px[k]); hiy = fmax(hiy, py[k]); hiz = fmax(hiz, pz[k]);
    }
    // group bounding box: its centre is the FP64 origin of the warp's FP32 frame
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lox = fmin(lox, __shfl_xor_sync(MHPC_FULL, lox, o));
        loy = fmin(loy, __shfl_xor_sync(MHPC_FULL, loy, o));
        loz = fmin(loz, __shfl_xor_sync(MHPC_FULL, loz, o));
        hix = fmax(hix, __shfl_xor_sync(MHPC_FULL, hix, o));
        hiy = fmax(hiy, __shfl_xor_sync(MHPC_FULL, hiy, o));
        hiz = fmax(hiz, __shfl_xor_sync(MHPC_FULL, hiz, o));
    }
    const double cx = 0.5 * (lox + hix), cy = 0.5 * (loy + hiy), cz = 0.5 * (loz + hiz);
    const float chx = (float)cx, chy = (float)cy, chz = (float)cz;
    const float clx = (float)(cx - (double)chx), cly = (float)(cy - (double)chy), clz = (float)(cz - (double)chz);
    float rx[PPL], ry[PPL], rz[PPL], e2[PPL], fax[PPL], fay[PPL], faz[PPL];
    double ax[PPL], ay[PPL], az[PPL];
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        // the particle's offset is formed exactly like its own leaf's, so the
        // self-interaction has R = 0 (a one-ulp mismatch would leave m R / eps^3)
        const int lf = __ldg(leaf_node + (valid[k] ? s[k] : (long)P.n - 1));
        const float4 hp = __ldg(wrec + 4 * (size_t)lf);
        const float4 lp = __ldg(wrec + 4 * (size_t)lf + 1);
        rx[k] = (hp.x - chx) + (lp.x - clx);
        ry[k] = (hp.y - chy) + (lp.y - cly);
        rz[k] = (hp.z - chz) + (lp.z - clz);
        e2[k] = (float)e2d[k];
        fax[k] = fay[k] = faz[k] = 0.f;
        ax[k] = ay[k] = az[k] = 0.0;
    }
    int since = 0;
    unsigned ninter = 0, nvisit = 0, nquad = 0;
    int nd = 0;
    while (nd < M) {
        const float4 hp = __ldg(wrec + 4 * (size_t)nd);
        const float4 lp = __ldg(wrec + 4 * (size_t)nd + 1);
        const int2 lk = __ldg(link + nd);
        ++nvisit;
        const float nx = (hp.x - chx) + (lp.x - clx);
        const float ny = (hp.y - chy) + (lp.y - cly);
        const float nz = (hp.z - chz) + (lp.z - clz);
        const bool leaf = lk.y & ND_LEAF;
        float Rx[PPL], Ry[PPL], Rz[PPL], r2[PPL];
        bool far = true;
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
            Rx[k] = rx[k] - nx; Ry[k] = ry[k] - ny; Rz[k] = rz[k] - nz;
            const float d2 = fmaf(Rx[k], Rx[k], fmaf(Ry[k], Ry[k], Rz[k] * Rz[k]));
            far = far && (!valid[k] || lp.w <= d2);
            r2[k] = d2 + e2[k];
        }
        if (!leaf && !__all_sync(MHPC_FULL, far)) { ++nd; continue; }
        float4 a0;
        float2 a1;
        if (!leaf) {
            a0 = __ldg(wrec + 4 * (size_t)nd + 2);
            const float4 a3 = __ldg(wrec + 4 * (size_t)nd + 3);
            a1 = make_float2(a3.x, a3.y);
            ++nquad;
        }
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
            const float ri = r2[k] > 0.f ? rsqrtf(r2[k]) : 0.f;
            const float ri2 = ri * ri;
            const float mri3 = hp.w * ri * ri2;
            fax[k] = fmaf(-mri3, Rx[k], fax[k]);
            fay[k] = fmaf(-mri3, Ry[k], fay[k]);
            faz[k] = fmaf(-mri3, Rz[k], faz[k]);
            if (!leaf) {
                const float qx = a0.x * Rx[k] + a0.y * Ry[k] + a0.z * Rz[k];
                const float qy = a0.y * Rx[k] + a0.w * Ry[k] + a1.x * Rz[k];
                const float qz = a0.z * Rx[k] + a1.x * Ry[k] + a1.y * Rz[k];
                const float rqr = qx * Rx[k] + qy * Ry[k] + qz * Rz[k];
                const float ri5 = ri2 * ri2 * ri;
                const float t = 2.5f * rqr * ri5 * ri2;
                fax[k] += qx * ri5 - t * Rx[k];
                fay[k] += qy * ri5 - t * Ry[k];
                faz[k] += qz * ri5 - t * Rz[k];
            }
        }
        ++ninter;
        if (++since == kFlush) {
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                ax[k] += fax[k]; ay[k] += fay[k]; az[k] += faz[k];
                fax[k] = fay[k] = faz[k] = 0.f;
            }
            since = 0;
        }
        nd = lk.x;
    }
    unsigned nv = 0;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        ax[k] += fax[k]; ay[k] += fay[k]; az[k] += faz[k];
        if (valid[k]) {
            const int o = __ldg(perm + s[k]);
            gax[o] = P.G * ax[k]; gay[o] = P.G * ay[k]; gaz[o] = P.G * az[k];
        }
        nv += __popc(__ballot_sync(MHPC_FULL, valid[k]));
    }
    if (lane == 0) {
        atomicAdd(&st->interactions, (unsigned long long)ninter * nv);
        atomicAdd(&st->nodes_visited, (unsigned long long)nvisit);
        atomicAdd(&st->quad_interactions, (unsigned long long)nquad * nv);
    }
}

// ------------------------------------------------- mixed, interaction lists
// One warp per group of kListGroup = 64 consecutive sorted particles (two per
// lane: members lane and 32 + lane).  The traversal is lane-parallel: each
// step pops up to 32 nodes from a per-warp stack in shared memory and every
// lane tests one node against the group's kListSub sub-boxes (bounding boxes
// of kListGroup / kListSub consecutive members).  A cell is accepted when
// edge^2/theta <= dist(com, box)^2 for every sub-box, i.e. for every member
// the cell subtends at most sqrt(theta) (edge over distance); accepted cells
// go to a cell list (monopole + quadrupole), particles to a leaf list
// (monopole), opened cells push their children.  Whenever a list holds 32
// entries or more the whole warp evaluates it: a branch-free loop over
// shared-memory entries, every lane applying each entry to its two
// particles, FP32 partial sums added into FP64 accumulators after each list.
// Positions are FP32 offsets from the group centre formed from the nodes'
// FP32 hi/lo split, particles taking their own leaf's values so that the
// self-interaction has R = 0 exactly.
//
// Stack bound: a pop of k nodes pushes at most 8k (cells with digit children;
// shared-key buckets are expanded straight into the leaf list), so k is
// limited to keep room for a depth-first descent (7 per level, 21 levels)
// on top of the current stack; the stack never overflows, a check that cannot
// fire reports MHPC_ERR_DEPTH instead of writing past it.
// particles per lane (2: groups of 64; 4: groups of 128, build-time choice)
#ifndef MHPC_LIST_PPL
#define MHPC_LIST_PPL 2
#endif
constexpr int kPPL = MHPC_LIST_PPL;
constexpr int kNP = kPPL / 2;  // particle pairs per lane (one paired FP32 instruction each)
constexpr int kListGroup = 32 * kPPL;
constexpr int kEvalUnroll = kPPL == 2 ? 8 : 4;
constexpr int kListSub = 8;
constexpr int kListStack = 1024;
constexpr int kListReserve = 7 * 22 + 8;
constexpr int kListCap = 64;

struct ListSmem {
    int stk[kListStack];
    float4 cpos[kListCap];  // cell: x, y, z (group frame), m
    float4 cq0[kListCap];   // cell: Qxx Qxy Qxz Qyy
    float2 cq1[kListCap];   // cell: Qyz Qzz
    float4 lpos[kListCap];  // leaf: x, y, z, m
    // sub-boxes, one array per component so that sub-boxes b, b+1 load as a
    // float2: lower corner, NEGATED upper corner, alpha |a|_min, quad_alpha |a|_min
    float bx0[kListSub], by0[kListSub], bz0[kListSub], bw0[kListSub];
    float nbx1[kListSub], nby1[kListSub], nbz1[kListSub], bw1[kListSub];
    int defer[32];
};

// kGuard: some softened distance may be 0 (eps2 = 0), so 1/r is guarded; with
// eps2 >= 1e-20 every r^2 >= eps2 keeps 1/r^3 finite and the guard is dropped
// (it costs 11 % of the walk's instructions).
// Packed form of the two evaluations for sm_100's paired FP32 instructions:
// a lane's two particles are the halves of a float2, so every multiply/add of
// the interaction is one paired instruction.  Each half is rounded exactly like
// the scalar form (same operations in the same order; negations are exact).
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 ld2(const float* a, int e) { return *reinterpret_cast<const float2*>(a + e); }

template <bool kGuard>
__device__ __forceinline__ float2 rsqrt2(float2 r2) {
    float2 ri;
    ri.x = kGuard ? (r2.x > 0.f ? rsqrtf(r2.x) : 0.f) : rsqrtf(r2.x);
    ri.y = kGuard ? (r2.y > 0.f ? rsqrtf(r2.y) : 0.f) : rsqrtf(r2.y);
    return ri;
}

template <bool kGuard>
__device__ __forceinline__ void eval_cells_x2(const ListSmem& S, int count, const float (&rx)[kPPL],
                                              const float (&ry)[kPPL], const float (&rz)[kPPL],
                                              const float (&e2)[kPPL], double (&ax)[kPPL], double (&ay)[kPPL],
                                              double (&az)[kPPL]) {
    float2 PX[kNP], PY[kNP], PZ[kNP], E2[kNP], fx[kNP], fy[kNP], fz[kNP];
#pragma unroll
    for (int q = 0; q < kNP; ++q) {
        PX[q] = make_float2(rx[2 * q], rx[2 * q + 1]); PY[q] = make_float2(ry[2 * q], ry[2 * q + 1]);
        PZ[q] = make_float2(rz[2 * q], rz[2 * q + 1]); E2[q] = make_float2(e2[2 * q], e2[2 * q + 1]);
        fx[q] = bc2(0.f); fy[q] = bc2(0.f); fz[q] = bc2(0.f);
    }
#pragma unroll kEvalUnroll
    for (int e = 0; e < count; ++e) {
        const float4 c = S.cpos[e];
        const float4 a0 = S.cq0[e];
        const float2 a1 = S.cq1[e];
#pragma unroll
        for (int q = 0; q < kNP; ++q) {
            const float2 Rx = __fadd2_rn(PX[q], bc2(-c.x)), Ry = __fadd2_rn(PY[q], bc2(-c.y)),
                         Rz = __fadd2_rn(PZ[q], bc2(-c.z));
            const float2 r2 = __ffma2_rn(Rx, Rx, __ffma2_rn(Ry, Ry, __ffma2_rn(Rz, Rz, E2[q])));
            const float2 ri = rsqrt2<kGuard>(r2);
            const float2 ri2 = __fmul2_rn(ri, ri);
            const float2 ri3 = __fmul2_rn(ri, ri2);
            const float2 ri5 = __fmul2_rn(ri3, ri2);
            const float2 qx = __ffma2_rn(bc2(a0.x), Rx, __ffma2_rn(bc2(a0.y), Ry, __fmul2_rn(bc2(a0.z), Rz)));
            const float2 qy = __ffma2_rn(bc2(a0.y), Rx, __ffma2_rn(bc2(a0.w), Ry, __fmul2_rn(bc2(a1.x), Rz)));
            const float2 qz = __ffma2_rn(bc2(a0.z), Rx, __ffma2_rn(bc2(a1.x), Ry, __fmul2_rn(bc2(a1.y), Rz)));
            const float2 rqr = __ffma2_rn(qx, Rx, __ffma2_rn(qy, Ry, __fmul2_rn(qz, Rz)));
            // -(m/r^3 + 5/2 RQR/r^7)
            const float2 cc =
                __ffma2_rn(bc2(-c.w), ri3, __fmul2_rn(__fmul2_rn(__fmul2_rn(bc2(-2.5f), rqr), ri5), ri2));
            fx[q] = __ffma2_rn(cc, Rx, __ffma2_rn(qx, ri5, fx[q]));
            fy[q] = __ffma2_rn(cc, Ry, __ffma2_rn(qy, ri5, fy[q]));
            fz[q] = __ffma2_rn(cc, Rz, __ffma2_rn(qz, ri5, fz[q]));
        }
    }
#pragma unroll
    for (int q = 0; q < kNP; ++q) {
        ax[2 * q] += fx[q].x; ay[2 * q] += fy[q].x; az[2 * q] += fz[q].x;
        ax[2 * q + 1] += fx[q].y; ay[2 * q + 1] += fy[q].y; az[2 * q + 1] += fz[q].y;
    }
}

template <bool kGuard>
__device__ __forceinline__ void eval_leaves_x2(const ListSmem& S, int count, const float (&rx)[kPPL],
                                               const float (&ry)[kPPL], const float (&rz)[kPPL],
                                               const float (&e2)[kPPL], double (&ax)[kPPL], double (&ay)[kPPL],
                                               double (&az)[kPPL]) {
    float2 PX[kNP], PY[kNP], PZ[kNP], E2[kNP], fx[kNP], fy[kNP], fz[kNP];
#pragma unroll
    for (int q = 0; q < kNP; ++q) {
        PX[q] = make_float2(rx[2 * q], rx[2 * q + 1]); PY[q] = make_float2(ry[2 * q], ry[2 * q + 1]);
        PZ[q] = make_float2(rz[2 * q], rz[2 * q + 1]); E2[q] = make_float2(e2[2 * q], e2[2 * q + 1]);
        fx[q] = bc2(0.f); fy[q] = bc2(0.f); fz[q] = bc2(0.f);
    }
#pragma unroll kEvalUnroll
    for (int e = 0; e < count; ++e) {
        const float4 c = S.lpos[e];
#pragma unroll
        for (int q = 0; q < kNP; ++q) {
            const float2 Rx = __fadd2_rn(PX[q], bc2(-c.x)), Ry = __fadd2_rn(PY[q], bc2(-c.y)),
                         Rz = __fadd2_rn(PZ[q], bc2(-c.z));
            const float2 r2 = __ffma2_rn(Rx, Rx, __ffma2_rn(Ry, Ry, __ffma2_rn(Rz, Rz, E2[q])));
            const float2 ri = rsqrt2<kGuard>(r2);
            const float2 nm = __fmul2_rn(bc2(-c.w), __fmul2_rn(__fmul2_rn(ri, ri), ri));  // -m / r^3
            fx[q] = __ffma2_rn(nm, Rx, fx[q]);
            fy[q] = __ffma2_rn(nm, Ry, fy[q]);
            fz[q] = __ffma2_rn(nm, Rz, fz[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < kNP; ++q) {
        ax[2 * q] += fx[q].x; ay[2 * q] += fy[q].x; az[2 * q] += fz[q].x;
        ax[2 * q + 1] += fx[q].y; ay[2 * q + 1] += fy[q].y; az[2 * q + 1] += fz[q].y;
    }
}

// kPot: also the potential, -(m/r + RQR/(2 r^5)) per cell and -m/r per leaf,
// leaving out the particle's own leaf (R = 0 exactly).
template <bool kGuard, bool kPot>
__device__ __forceinline__ void eval_cells(const ListSmem& S, int count, const float (&rx)[kPPL], const float (&ry)[kPPL],
                                           const float (&rz)[kPPL], const float (&e2)[kPPL], double (&ax)[kPPL],
                                           double (&ay)[kPPL], double (&az)[kPPL], double (&ph)[kPPL]) {
    float fx[kPPL] = {}, fy[kPPL] = {}, fz[kPPL] = {}, fp[kPPL] = {};
#pragma unroll kEvalUnroll
    for (int e = 0; e < count; ++e) {
        const float4 c = S.cpos[e];
        const float4 a0 = S.cq0[e];
        const float2 a1 = S.cq1[e];
#pragma unroll
        for (int k = 0; k < kPPL; ++k) {
            const float Rx = rx[k] - c.x, Ry = ry[k] - c.y, Rz = rz[k] - c.z;
            const float r2 = fmaf(Rx, Rx, fmaf(Ry, Ry, fmaf(Rz, Rz, e2[k])));
            const float ri = kGuard ? (r2 > 0.f ? rsqrtf(r2) : 0.f) : rsqrtf(r2);
            const float ri2 = ri * ri;
            const float ri3 = ri * ri2;
            const float ri5 = ri3 * ri2;
            const float qx = fmaf(a0.x, Rx, fmaf(a0.y, Ry, a0.z * Rz));
            const float qy = fmaf(a0.y, Rx, fmaf(a0.w, Ry, a1.x * Rz));
            const float qz = fmaf(a0.z, Rx, fmaf(a1.x, Ry, a1.y * Rz));
            const float rqr = fmaf(qx, Rx, fmaf(qy, Ry, qz * Rz));
            // -(m/r^3 + 5/2 RQR/r^7) R + Q R / r^5
            const float cc = -fmaf(c.w, ri3, 2.5f * rqr * ri5 * ri2);
            fx[k] = fmaf(cc, Rx, fmaf(qx, ri5, fx[k]));
            fy[k] = fmaf(cc, Ry, fmaf(qy, ri5, fy[k]));
            fz[k] = fmaf(cc, Rz, fmaf(qz, ri5, fz[k]));
            if (kPot) fp[k] -= fmaf(c.w, ri, 0.5f * rqr * ri5);
        }
    }
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
        ax[k] += fx[k]; ay[k] += fy[k]; az[k] += fz[k];
        if (kPot) ph[k] += fp[k];
    }
}

template <bool kGuard, bool kPot>
__device__ __forceinline__ void eval_leaves(const ListSmem& S, int count, const float (&rx)[kPPL], const float (&ry)[kPPL],
                                            const float (&rz)[kPPL], const float (&e2)[kPPL], double (&ax)[kPPL],
                                            double (&ay)[kPPL], double (&az)[kPPL], double (&ph)[kPPL]) {
    float fx[kPPL] = {}, fy[kPPL] = {}, fz[kPPL] = {}, fp[kPPL] = {};
#pragma unroll kEvalUnroll
    for (int e = 0; e < count; ++e) {
        const float4 c = S.lpos[e];
#pragma unroll
        for (int k = 0; k < kPPL; ++k) {
            const float Rx = rx[k] - c.x, Ry = ry[k] - c.y, Rz = rz[k] - c.z;
            const float r2 = fmaf(Rx, Rx, fmaf(Ry, Ry, fmaf(Rz, Rz, e2[k])));
            const float ri = kGuard ? (r2 > 0.f ? rsqrtf(r2) : 0.f) : rsqrtf(r2);
            const float mri3 = c.w * (ri * ri * ri);
            fx[k] = fmaf(-mri3, Rx, fx[k]);
            fy[k] = fmaf(-mri3, Ry, fy[k]);
            fz[k] = fmaf(-mri3, Rz, fz[k]);
            if (kPot) fp[k] -= (Rx == 0.f && Ry == 0.f && Rz == 0.f) ? 0.f : c.w * ri;
        }
    }
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
        ax[k] += fx[k]; ay[k] += fy[k]; az[k] += fz[k];
        if (kPot) ph[k] += fp[k];
    }
}

// the packed forms for the force walk, the scalar forms when the potential is wanted
constexpr bool kPackedEval = true;
template <bool kGuard, bool kPot>
__device__ __forceinline__ void eval_cells_sel(const ListSmem& S, int count, const float (&rx)[kPPL], const float (&ry)[kPPL],
                                               const float (&rz)[kPPL], const float (&e2)[kPPL], double (&ax)[kPPL],
                                               double (&ay)[kPPL], double (&az)[kPPL], double (&ph)[kPPL]) {
    if (kPackedEval && !kPot) eval_cells_x2<kGuard>(S, count, rx, ry, rz, e2, ax, ay, az);
    else eval_cells<kGuard, kPot>(S, count, rx, ry, rz, e2, ax, ay, az, ph);
}
template <bool kGuard, bool kPot>
__device__ __forceinline__ void eval_leaves_sel(const ListSmem& S, int count, const float (&rx)[kPPL], const float (&ry)[kPPL],
                                                const float (&rz)[kPPL], const float (&e2)[kPPL], double (&ax)[kPPL],
                                                double (&ay)[kPPL], double (&az)[kPPL], double (&ph)[kPPL]) {
    if (kPackedEval && !kPot) eval_leaves_x2<kGuard>(S, count, rx, ry, rz, e2, ax, ay, az);
    else eval_leaves<kGuard, kPot>(S, count, rx, ry, rz, e2, ax, ay, az, ph);
}

constexpr int kListBlock = 128;
// relative rule: a sub-box's smallest previous |a| is taken as at least this
// fraction of its largest (the oracle's statement uses the same floor)
constexpr float kRelFloor = 0.1f;
// Resident blocks per SM the list walk is compiled for: 5 (96 registers, no
// spills in the force walk) measured 3 % faster at 16.7 M than the
// unconstrained 116 registers (4 blocks); 6 blocks (80 registers) spill and
// run 1-2 % slower than 4.
#ifndef MHPC_LISTS_MIN_BLOCKS
#define MHPC_LISTS_MIN_BLOCKS 5
#endif

template <bool kGuard, bool kRel, bool kPot>
__global__ void __launch_bounds__(kListBlock, MHPC_LISTS_MIN_BLOCKS) k_grav_lists(TreeDev T, GravParams P,
                                                                                 const double* __restrict__ sx,
                                                           const double* __restrict__ sy,
                                                           const double* __restrict__ sz,
                                                           const double* __restrict__ sh,
                                                           const int* __restrict__ perm, double* __restrict__ gax,
                                                           double* __restrict__ gay, double* __restrict__ gaz,
                                                           DevStatus* st) {
    __shared__ ListSmem smem[kListBlock / 32];
    if (st->code) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    ListSmem& S = smem[threadIdx.x >> 5];
    const long gwarp = ((long)blockIdx.x * kListBlock + threadIdx.x) >> 5;
    const long ngroups = ((long)P.n + kListGroup - 1) / kListGroup;
    if (gwarp >= ngroups) return;
    const long s0 = gwarp * kListGroup;
    long s[kPPL];
    bool valid[kPPL];
    int sl[kPPL];
    float e2[kPPL];
    double lox = 1e300, loy = 1e300, loz = 1e300, hix = -1e300, hiy = -1e300, hiz = -1e300;
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
        s[k] = s0 + k * 32 + lane;
        valid[k] = s[k] < P.n;
        sl[k] = (int)(valid[k] ? s[k] : (long)P.n - 1);
        const double px = __ldg(sx + sl[k]), py = __ldg(sy + sl[k]), pz = __ldg(sz + sl[k]);
        double e = P.eps2;
        if (P.h_factor > 0.0) {
            // softening tied to h: at least 1e-20 (h >= 2e-10 h_factor^-1 in
            // practice), so that every r^2 >= eps^2 keeps 1/r^3 finite and the
            // walk runs without the r^2 = 0 guard
            const double hh = P.h_factor * __ldg(sh + sl[k]);
            e = fmax(e + hh * hh, 1e-20);
        }
        e2[k] = (float)e;
        lox = fmin(lox, px); loy = fmin(loy, py); loz = fmin(loz, pz);
        hix = fmax(hix, px); hiy = fmax(hiy, py); hiz = fmax(hiz, pz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lox = fmin(lox, __shfl_xor_sync(MHPC_FULL, lox, o));
        loy = fmin(loy, __shfl_xor_sync(MHPC_FULL, loy, o));
        loz = fmin(loz, __shfl_xor_sync(MHPC_FULL, loz, o));
        hix = fmax(hix, __shfl_xor_sync(MHPC_FULL, hix, o));
        hiy = fmax(hiy, __shfl_xor_sync(MHPC_FULL, hiy, o));
        hiz = fmax(hiz, __shfl_xor_sync(MHPC_FULL, hiz, o));
    }
    const double cx = 0.5 * (lox + hix), cy = 0.5 * (loy + hiy), cz = 0.5 * (loz + hiz);
    const float chx = (float)cx, chy = (float)cy, chz = (float)cz;
    const float clx = (float)(cx - (double)chx), cly = (float)(cy - (double)chy), clz = (float)(cz - (double)chz);
    float rx[kPPL], ry[kPPL], rz[kPPL];
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
        const int lf = __ldg(T.leaf_node + sl[k]);
        const float4 hp = __ldg(T.wrec + 4 * (size_t)lf);
        const float4 lp = __ldg(T.wrec + 4 * (size_t)lf + 1);
        rx[k] = (hp.x - chx) + (lp.x - clx);
        ry[k] = (hp.y - chy) + (lp.y - cly);
        rz[k] = (hp.z - chz) + (lp.z - clz);
        // sub-box of members [4 kPPL b, 4 kPPL (b + 1)): 4 kPPL-lane segments of member row k;
        // relative rule: alpha times the smallest previous |a| of the sub-box
        // (read before this walk overwrites the accelerations), floored at
        // kRelFloor times the largest: near a potential minimum |a| tends to
        // zero, and without the floor such a group would open the whole tree
        float amin = 0.f, amax = 0.f;
        const float qratio = kRel ? (float)(P.quad_alpha / P.rel_alpha) : 0.f;
        if (kRel) {
            const int o = __ldg(perm + sl[k]);
            const double gx = gax[o], gy = gay[o], gz = gaz[o];
            amin = (float)(P.rel_alpha * sqrt(gx * gx + gy * gy + gz * gz));
            amax = amin;
        }
        float bx0 = rx[k], by0 = ry[k], bz0 = rz[k], bx1 = rx[k], by1 = ry[k], bz1 = rz[k];
#pragma unroll
        for (int o = 2 * kPPL; o > 0; o >>= 1) {
            bx0 = fminf(bx0, __shfl_xor_sync(MHPC_FULL, bx0, o));
            by0 = fminf(by0, __shfl_xor_sync(MHPC_FULL, by0, o));
            bz0 = fminf(bz0, __shfl_xor_sync(MHPC_FULL, bz0, o));
            bx1 = fmaxf(bx1, __shfl_xor_sync(MHPC_FULL, bx1, o));
            by1 = fmaxf(by1, __shfl_xor_sync(MHPC_FULL, by1, o));
            if (kRel) amin = fminf(amin, __shfl_xor_sync(MHPC_FULL, amin, o));
            if (kRel) amax = fmaxf(amax, __shfl_xor_sync(MHPC_FULL, amax, o));
            bz1 = fmaxf(bz1, __shfl_xor_sync(MHPC_FULL, bz1, o));
        }
        if (kRel) amin = fmaxf(amin, kRelFloor * amax);
        if ((lane & (4 * kPPL - 1)) == 0) {
            const int b = k * (8 / kPPL) + lane / (4 * kPPL);
            S.bx0[b] = bx0; S.by0[b] = by0; S.bz0[b] = bz0; S.bw0[b] = amin;
            // bhi.w: quad_alpha |a|_min of the sub-box (monopole threshold)
            S.nbx1[b] = -bx1; S.nby1[b] = -by1; S.nbz1[b] = -bz1; S.bw1[b] = kRel ? amin * qratio : 0.f;
        }
    }
    const double edge0 = ord_to_dbl(P.ord[1]) - ord_to_dbl(P.ord[0]);
    const float edge2 = (float)(edge0 * edge0);
    // the root's children: node 0 and its skip chain
    int top = 0;
    if (lane == 0) {
        int c = 0;
        while (c < M && top < 8) { S.stk[top++] = c; c = __ldg(&T.link[c].x); }
        if (c < M) set_status(st, MHPC_ERR_DEPTH, 1);
    }
    top = __shfl_sync(MHPC_FULL, top, 0);
    __syncwarp();
    double ax[kPPL] = {}, ay[kPPL] = {}, az[kPPL] = {}, ph[kPPL] = {};
    int ncell = 0, nleaf = 0;
    unsigned long long tested = 0, ncell_tot = 0, nleaf_tot = 0;
    while (top > 0) {
        int room = (kListStack - kListReserve - top) / 7;
        int k = top < 32 ? top : 32;
        if (k > room) k = room > 1 ? room : 1;
        const bool act = lane < k;
        const int nd = act ? S.stk[top - 1 - lane] : 0;
        __syncwarp();
        top -= k;
        tested += k;
        bool acc_leaf = false, acc_cell = false, open = false;
        float nx = 0.f, ny = 0.f, nz = 0.f, m = 0.f;
        float4 w2 = make_float4(0.f, 0.f, 0.f, 0.f), w3 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (act) {
            // the node's whole record (one 64-byte line): position, criterion,
            // quadrupole and child mask arrive in one round trip
            const float4* w = T.wrec + 4 * (size_t)nd;
            const float4 hp = __ldg(w);
            const float4 lp = __ldg(w + 1);
            w2 = __ldg(w + 2);
            w3 = __ldg(w + 3);
            const int bits = __float_as_int(w3.z);
            const int info = bits & 0x1ff;
            nx = (hp.x - chx) + (lp.x - clx);
            ny = (hp.y - chy) + (lp.y - cly);
            nz = (hp.z - chz) + (lp.z - clz);
            m = hp.w;
            if (info & ND_LEAF) {
                acc_leaf = true;
            } else {
                // kRel: squared edge of the cell, edge0^2 / 4^level (exact power of two)
                const float l2 = kRel ? edge2 * __int_as_float((127 - 2 * (info & 0xff)) << 23) : 0.f;
                bool ok = true;
                // relative rule: the quadrupole term M l^2 / d^4 below
                // quad_alpha |a| for every sub-box makes the cell a monopole
                bool mono = kRel;
                const float ml2 = m * l2;
                // sub-boxes in pairs on paired FP32 instructions (each half rounded
                // like the scalar form); the max/compare steps stay scalar
                const float2 NX = bc2(nx), NY = bc2(ny), NZ = bc2(nz), MNX = bc2(-nx), MNY = bc2(-ny), MNZ = bc2(-nz);
#pragma unroll
                for (int b = 0; b < kListSub; b += 2) {
                    const float2 ax0 = __fadd2_rn(ld2(S.bx0, b), MNX), ax1 = __fadd2_rn(NX, ld2(S.nbx1, b));
                    const float2 ay0 = __fadd2_rn(ld2(S.by0, b), MNY), ay1 = __fadd2_rn(NY, ld2(S.nby1, b));
                    const float2 az0 = __fadd2_rn(ld2(S.bz0, b), MNZ), az1 = __fadd2_rn(NZ, ld2(S.nbz1, b));
                    const float2 dx = make_float2(fmaxf(fmaxf(ax0.x, ax1.x), 0.f), fmaxf(fmaxf(ax0.y, ax1.y), 0.f));
                    const float2 dy = make_float2(fmaxf(fmaxf(ay0.x, ay1.x), 0.f), fmaxf(fmaxf(ay0.y, ay1.y), 0.f));
                    const float2 dz = make_float2(fmaxf(fmaxf(az0.x, az1.x), 0.f), fmaxf(fmaxf(az0.y, az1.y), 0.f));
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                    if (kRel) {
                        // safety bound d >= l, then M l^3 <= alpha |a| d^5
                        // (d2 = 0 gives NaN: not accepted)
                        const float2 d4 = __fmul2_rn(d2, d2);
                        const float2 d1 = __fmul2_rn(d2, make_float2(rsqrtf(d2.x), rsqrtf(d2.y)));
                        const float2 lim = __fmul2_rn(__fmul2_rn(ld2(S.bw0, b), d4), d1);
                        const float2 qlim = __fmul2_rn(ld2(S.bw1, b), d4);
                        ok = ok && l2 <= d2.x && l2 <= d2.y && w3.w <= lim.x && w3.w <= lim.y;
                        mono = mono && ml2 <= qlim.x && ml2 <= qlim.y;
                    } else {
                        ok = ok && lp.w <= d2.x && lp.w <= d2.y;
                    }
                }
                // accepted monopoles go to the leaf list (monopole evaluation)
                acc_leaf = ok && mono;
                acc_cell = ok && !mono;
                open = !ok;
            }
        }
        const unsigned bl = __ballot_sync(MHPC_FULL, acc_leaf);
        if (acc_leaf) S.lpos[nleaf + __popc(bl & lt)] = make_float4(nx, ny, nz, m);
        nleaf += __popc(bl);
        const unsigned bc = __ballot_sync(MHPC_FULL, acc_cell);
        if (acc_cell) {
            const int i = ncell + __popc(bc & lt);
            S.cpos[i] = make_float4(nx, ny, nz, m);
            S.cq0[i] = w2;
            S.cq1[i] = make_float2(w3.x, w3.y);
        }
        ncell += __popc(bc);
        const int mask = open ? (__float_as_int(w3.z) >> 9) : 0;
        const bool bucket = open && (mask & 0x100);
        const unsigned bb = __ballot_sync(MHPC_FULL, bucket);
        if (bucket) S.defer[__popc(bb & lt)] = nd;
        const int nkid = (open && !bucket) ? __popc(mask & 0xff) : 0;
        int incl = nkid;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(MHPC_FULL, incl, 31);
        if (top + total > kListStack) {
            // unreachable by the bound on k; stop instead of overrunning
            if (lane == 0) set_status(st, MHPC_ERR_DEPTH, 2);
            return;
        }
        if (nkid) {
            const int4 k0 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd));
            const int4 k1 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd) + 1);
            const int all[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
            int w = top + incl - nkid;
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((mask >> d) & 1) S.stk[w++] = all[d];
        }
        top += total;
        __syncwarp();
        if (ncell >= 32) {
            eval_cells_sel<kGuard, kPot>(S, ncell, rx, ry, rz, e2, ax, ay, az, ph);
            ncell_tot += ncell;
            ncell = 0;
            __syncwarp();
        }
        if (nleaf >= 32) {
            eval_leaves_sel<kGuard, kPot>(S, nleaf, rx, ry, rz, e2, ax, ay, az, ph);
            nleaf_tot += nleaf;
            nleaf = 0;
            __syncwarp();
        }
        // shared-key buckets: their children are consecutive leaves (the
        // leaf list holds fewer than 32 entries here, at most 63 after a round)
        const int ndefer = __popc(bb);
        for (int d = 0; d < ndefer; ++d) {
            const int b = S.defer[d];
            const int end = __ldg(&T.link[b].x);
            for (int c0 = b + 1; c0 < end; c0 += 32) {
                const int c = c0 + lane;
                const bool a = c < end;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (a) {
                    const float4 hp = __ldg(T.wrec + 4 * (size_t)c);
                    const float4 lp = __ldg(T.wrec + 4 * (size_t)c + 1);
                    v = make_float4((hp.x - chx) + (lp.x - clx), (hp.y - chy) + (lp.y - cly),
                                    (hp.z - chz) + (lp.z - clz), hp.w);
                }
                const unsigned ba = __ballot_sync(MHPC_FULL, a);
                if (a) S.lpos[nleaf + __popc(ba & lt)] = v;
                nleaf += __popc(ba);
                __syncwarp();
                if (nleaf >= 32) {
                    eval_leaves_sel<kGuard, kPot>(S, nleaf, rx, ry, rz, e2, ax, ay, az, ph);
                    nleaf_tot += nleaf;
                    nleaf = 0;
                    __syncwarp();
                }
            }
        }
    }
    if (ncell) eval_cells_sel<kGuard, kPot>(S, ncell, rx, ry, rz, e2, ax, ay, az, ph);
    if (nleaf) eval_leaves_sel<kGuard, kPot>(S, nleaf, rx, ry, rz, e2, ax, ay, az, ph);
    ncell_tot += ncell;
    nleaf_tot += nleaf;
    unsigned nv = 0;
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
        if (valid[k]) {
            const int o = __ldg(perm + s[k]);
            gax[o] = P.G * ax[k]; gay[o] = P.G * ay[k]; gaz[o] = P.G * az[k];
            if (kPot) P.pot[o] = P.G * ph[k];
        }
        nv += __popc(__ballot_sync(MHPC_FULL, valid[k]));
    }
    if (lane == 0) {
        atomicAdd(&st->interactions, (ncell_tot + nleaf_tot) * nv);
        atomicAdd(&st->nodes_visited, tested);
        atomicAdd(&st->quad_interactions, ncell_tot * nv);
    }
}

}  // namespace

int gravity_v2(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
               const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
               cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    long groups = ((long)P.n + 31) / 32;
    long blocks = (groups * 32 + kWalkBlock - 1) / kWalkBlock;
    k_grav_v2<<<(int)blocks, kWalkBlock, 0, s>>>(T.com, T.link, T.nodes, P, sx, sy, sz, sh, perm, gax, gay, gaz, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int gravity_v1(const TreeDev& T, const GravParams& P, const double* sh, const int* perm, double* gax, double* gay,
               double* gaz, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    const long blocks = ((long)P.n + kWalkBlock - 1) / kWalkBlock;
    k_grav_v1<<<(int)blocks, kWalkBlock, 0, s>>>(T.com, T.link, T.nodes, T.leaf_node, P, sh, perm, gax, gay, gaz, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int gravity_mixed(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
                  const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
                  cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    constexpr int PPL = MHPC_MIXED_PPL;
    long groups = ((long)P.n + 32 * PPL - 1) / (32 * PPL);
    long blocks = (groups * 32 + kWalkBlock - 1) / kWalkBlock;
    k_grav_mixed<PPL><<<(int)blocks, kWalkBlock, 0, s>>>(T.wrec, T.link, T.nodes, T.leaf_node, P, sx,
                                                         sy, sz, sh, perm, gax, gay, gaz, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int gravity_lists(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
                  const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
                  cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    const long groups = ((long)P.n + kListGroup - 1) / kListGroup;
    const long blocks = (groups * 32 + kListBlock - 1) / kListBlock;
    // the self-interaction has R = 0 and r^2 = eps2: 1/r^3 stays finite in
    // FP32 for eps2 >= 1e-20
    const bool guard = !(P.eps2 >= 1e-20) && !(P.h_factor > 0.0), rel = P.rel_alpha > 0.0;
#define MHPC_LISTS(G_, R_, P_) \
    k_grav_lists<G_, R_, P_><<<(int)blocks, kListBlock, 0, s>>>(T, P, sx, sy, sz, sh, perm, gax, gay, gaz, st)
    if (P.pot) {
        // potential (diagnostics): separate instantiations, the force walk stays as it is
        if (!guard && !rel) MHPC_LISTS(false, false, true);
        else if (!guard && rel) MHPC_LISTS(false, true, true);
        else if (guard && !rel) MHPC_LISTS(true, false, true);
        else MHPC_LISTS(true, true, true);
    } else {
        if (!guard && !rel) MHPC_LISTS(false, false, false);
        else if (!guard && rel) MHPC_LISTS(false, true, false);
        else if (guard && !rel) MHPC_LISTS(true, false, false);
        else MHPC_LISTS(true, true, false);
    }
#undef MHPC_LISTS
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
