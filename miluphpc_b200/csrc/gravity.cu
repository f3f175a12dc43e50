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

// -------------------------------------------------------------- mixed FP32
// The group's centre c (FP64, centre of its bounding box) is subtracted once;
// lanes hold their position relative to c in FP32, nodes are stored as
// float hi + float lo of the FP64 centre of mass, so node - c is formed as
// (hi - c_hi) + (lo - c_lo) without losing the digits that FP32 absolute
// coordinates would drop.  A cell is accepted for the warp when every lane
// has edge^2/theta <= |node - p|^2 + eps2 (the squared-ratio criterion with
// computeForces_v2's warp vote, applied at every level); accepted cells add
// monopole + quadrupole terms.  A box test per group would be cheaper per
// node but opens the whole interior of a group box that straddles a curve
// jump (Lebesgue order), which leaves single warps with tens of thousands of
// leaf interactions; the per-lane vote keeps the cost of such a group at the
// union of its parts.  FP32 partial sums are flushed into FP64 every kFlush
// accepted nodes (compensated accumulation).
constexpr int kFlush = 64;

__global__ void __launch_bounds__(kWalkBlock) k_grav_mixed(const float4* __restrict__ mpos, const float4* __restrict__ mlo,
                                                           const float4* __restrict__ q0, const float2* __restrict__ q1,
                                                           const int2* __restrict__ link, const int* __restrict__ nodes_total,
                                                           GravParams P, const double* __restrict__ sx,
                                                           const double* __restrict__ sy, const double* __restrict__ sz,
                                                           const double* __restrict__ sh, const int* __restrict__ perm,
                                                           double* __restrict__ gax, double* __restrict__ gay,
                                                           double* __restrict__ gaz, DevStatus* st) {
    if (st->code) return;
    const int M = *nodes_total;
    const int lane = threadIdx.x & 31;
    const long gwarp = ((long)blockIdx.x * kWalkBlock + threadIdx.x) >> 5;
    const long ngroups = ((long)P.n + 31) >> 5;
    if (gwarp >= ngroups) return;
    const long s0 = gwarp * 32;
    const long s = s0 + lane;
    const bool valid = s < P.n;
    const long sl = valid ? s : (long)P.n - 1;
    const double px = __ldg(sx + sl), py = __ldg(sy + sl), pz = __ldg(sz + sl);
    double e2d = P.eps2;
    if (P.h_factor > 0.0) { double e = P.h_factor * __ldg(sh + sl); e2d += e * e; }
    // group bounding box: its centre is the FP64 origin of the warp's FP32 frame
    double lox = px, loy = py, loz = pz, hix = px, hiy = py, hiz = pz;
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
    const float rx = (float)(px - cx), ry = (float)(py - cy), rz = (float)(pz - cz);
    const float e2 = (float)e2d;
    float fax = 0.f, fay = 0.f, faz = 0.f;
    double ax = 0.0, ay = 0.0, az = 0.0;
    int since = 0;
    unsigned long long ninter = 0, nvisit = 0, nquad = 0;
    int nd = 0;
    while (nd < M) {
        const float4 hp = __ldg(mpos + nd);
        const float4 lp = __ldg(mlo + nd);
        const int2 lk = __ldg(link + nd);
        ++nvisit;
        const float nx = (hp.x - chx) + (lp.x - clx);
        const float ny = (hp.y - chy) + (lp.y - cly);
        const float nz = (hp.z - chz) + (lp.z - clz);
        const bool leaf = lk.y & ND_LEAF;
        const float Rx = rx - nx, Ry = ry - ny, Rz = rz - nz;
        const float r2 = fmaf(Rx, Rx, fmaf(Ry, Ry, fmaf(Rz, Rz, e2)));
        if (!leaf && !__all_sync(MHPC_FULL, !valid || lp.w <= r2)) { ++nd; continue; }
        const float ri = r2 > 0.f ? rsqrtf(r2) : 0.f;
        const float ri2 = ri * ri;
        const float mri3 = hp.w * ri * ri2;
        fax = fmaf(-mri3, Rx, fax);
        fay = fmaf(-mri3, Ry, fay);
        faz = fmaf(-mri3, Rz, faz);
        if (!leaf) {
            ++nquad;
            const float4 a0 = __ldg(q0 + nd);
            const float2 a1 = __ldg(q1 + nd);
            const float qx = a0.x * Rx + a0.y * Ry + a0.z * Rz;
            const float qy = a0.y * Rx + a0.w * Ry + a1.x * Rz;
            const float qz = a0.z * Rx + a1.x * Ry + a1.y * Rz;
            const float rqr = qx * Rx + qy * Ry + qz * Rz;
            const float ri5 = ri2 * ri2 * ri;
            const float t = 2.5f * rqr * ri5 * ri2;
            fax += qx * ri5 - t * Rx;
            fay += qy * ri5 - t * Ry;
            faz += qz * ri5 - t * Rz;
        }
        ++ninter;
        if (++since == kFlush) {
            ax += fax; ay += fay; az += faz;
            fax = fay = faz = 0.f;
            since = 0;
        }
        nd = lk.x;
    }
    ax += fax; ay += fay; az += faz;
    if (valid) {
        const int o = __ldg(perm + s);
        gax[o] = P.G * ax; gay[o] = P.G * ay; gaz[o] = P.G * az;
    }
    unsigned nv = __popc(__ballot_sync(MHPC_FULL, valid));
    if (lane == 0) {
        atomicAdd(&st->interactions, ninter * nv);
        atomicAdd(&st->nodes_visited, nvisit);
        atomicAdd(&st->quad_interactions, nquad * nv);
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

int gravity_mixed(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
                  const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
                  cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    long groups = ((long)P.n + 31) / 32;
    long blocks = (groups * 32 + kWalkBlock - 1) / kWalkBlock;
    k_grav_mixed<<<(int)blocks, kWalkBlock, 0, s>>>(T.mpos, T.mlo, T.quad0, T.quad1, T.link, T.nodes, P, sx, sy, sz,
                                                    sh, perm, gax, gay, gaz, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
