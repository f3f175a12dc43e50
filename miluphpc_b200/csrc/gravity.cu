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

// PPL particles per lane: a warp takes 32 * PPL consecutive sorted particles;
// each visited node is loaded, placed in the warp frame and voted on once for
// all of them, which amortises the per-node instructions over PPL
// interactions (the kernel is issue-bound, not memory-bound).
template <int PPL>
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
        rx[k] = (float)(px[k] - cx); ry[k] = (float)(py[k] - cy); rz[k] = (float)(pz[k] - cz);
        e2[k] = (float)e2d[k];
        fax[k] = fay[k] = faz[k] = 0.f;
        ax[k] = ay[k] = az[k] = 0.0;
    }
    int since = 0;
    unsigned ninter = 0, nvisit = 0, nquad = 0;
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
        float Rx[PPL], Ry[PPL], Rz[PPL], r2[PPL];
        bool far = true;
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
            Rx[k] = rx[k] - nx; Ry[k] = ry[k] - ny; Rz[k] = rz[k] - nz;
            r2[k] = fmaf(Rx[k], Rx[k], fmaf(Ry[k], Ry[k], fmaf(Rz[k], Rz[k], e2[k])));
            far = far && (!valid[k] || lp.w <= r2[k]);
        }
        if (!leaf && !__all_sync(MHPC_FULL, far)) { ++nd; continue; }
        float4 a0;
        float2 a1;
        if (!leaf) { a0 = __ldg(q0 + nd); a1 = __ldg(q1 + nd); ++nquad; }
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
    constexpr int PPL = MHPC_MIXED_PPL;
    long groups = ((long)P.n + 32 * PPL - 1) / (32 * PPL);
    long blocks = (groups * 32 + kWalkBlock - 1) / kWalkBlock;
    k_grav_mixed<PPL><<<(int)blocks, kWalkBlock, 0, s>>>(T.mpos, T.mlo, T.quad0, T.quad1, T.link, T.nodes, P, sx,
                                                         sy, sz, sh, perm, gax, gay, gaz, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
