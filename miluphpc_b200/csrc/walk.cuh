// One-particle-per-warp neighbour walk shared by the sparse neighbour counts
// of the variable-h iteration and the neighbour-band repair.
#pragma once
#include "sph.cuh"

constexpr int kWalkStack = 512;
constexpr int kWalkReserve = 7 * 22 + 8;
constexpr int kWalkSmall = 16;   // cells with at most this many particles are tested whole

// One particle per warp (all 32 lanes call this; a lane that is not `valid`
// walks nothing but takes part in the warp's votes).  Visits every particle
// j of the leaves, small cells and shared-key buckets whose box comes within
// `rad` of the particle and whose largest h below the node reaches it:
// visit(j) is called on one lane per candidate (j may be the particle itself).
// Pruning is conservative (FP32 boxes rounded outward), so every j with
// d < rad and d < h_j is visited.  The walks here serve few, often far-reaching
// particles, so a whole warp pops up to 32 nodes per step; stack bound as in
// the other walks: a pop of k nodes pushes at most 8k, and k is limited so
// that a depth-first descent (7 per level, 22 levels) always fits on top.
template <class Visit>
__device__ __forceinline__ void warp_walk(const TreeDev& T, int M, bool valid, double px, double py, double pz,
                                          double rad, const float* __restrict__ node_hmax, int* S, int* RF, int* RE,
                                          DevStatus* st, Visit& visit) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    if (!__any_sync(MHPC_FULL, valid)) return;
    const float lx = __double2float_rd(px - rad), ly = __double2float_rd(py - rad), lz = __double2float_rd(pz - rad);
    const float ux = __double2float_ru(px + rad), uy = __double2float_ru(py + rad), uz = __double2float_ru(pz + rad);
    const float fx0 = __double2float_rd(px), fy0 = __double2float_rd(py), fz0 = __double2float_rd(pz);
    const float fx1 = __double2float_ru(px), fy1 = __double2float_ru(py), fz1 = __double2float_ru(pz);
    int top = 0;
    if (lane == 0) {
        int c = 0;
        while (c < M && top < 8) { S[top++] = c; c = __ldg(&T.link[c].x); }
        if (c < M) set_status(st, MHPC_ERR_DEPTH, 7);
    }
    top = __shfl_sync(MHPC_FULL, top, 0);
    __syncwarp();
    while (top > 0) {
        const int room = (kWalkStack - kWalkReserve - top) / 7;
        int kk = top < 32 ? top : 32;
        if (kk > room) kk = room > 1 ? room : 1;
        const bool act = lane < kk;
        const int nd = act ? S[top - 1 - lane] : 0;
        __syncwarp();
        top -= kk;
        int rf = 0, rlen = 0, kmask = 0;
        if (act) {
            const int2 lk = __ldg(T.link + nd);
            const float4 bl = __ldg(T.bmin + nd), bh = __ldg(T.bmax + nd);
            const float hn = __ldg(node_hmax + nd);
            const bool overlap =
                !(bh.x < lx || bl.x > ux || bh.y < ly || bl.y > uy || bh.z < lz || bl.z > uz) &&
                !(__fadd_ru(bh.x, hn) < fx0 || __fadd_rd(bl.x, -hn) > fx1 || __fadd_ru(bh.y, hn) < fy0 ||
                  __fadd_rd(bl.y, -hn) > fy1 || __fadd_ru(bh.z, hn) < fz0 || __fadd_rd(bl.z, -hn) > fz1);
            if (overlap) {
                rf = __ldg(T.first + nd);
                if (lk.y & ND_LEAF) {
                    rlen = 1;
                } else {
                    const int l = __ldg(T.last + nd);
                    const int km = __ldg(T.kmask + nd);
                    if (l - rf + 1 <= kWalkSmall || (km & 0x100)) rlen = l - rf + 1;
                    else kmask = km & 0xff;
                }
            }
        }
        const int nkid = __popc(kmask);
        int incl = nkid;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(MHPC_FULL, incl, 31);
        if (top + total > kWalkStack) {  // unreachable by the bound on kk
            if (lane == 0) set_status(st, MHPC_ERR_DEPTH, 8);
            return;
        }
        if (nkid) {
            const int4 k0 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd));
            const int4 k1 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd) + 1);
            const int all[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
            int wpos = top + incl - nkid;
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((kmask >> d) & 1) S[wpos++] = all[d];
        }
        top += total;
        // candidate ranges of this step with running ends
        int rincl = rlen;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, rincl, o);
            if (lane >= o) rincl += v;
        }
        const int ncand = __shfl_sync(MHPC_FULL, rincl, 31);
        const unsigned br = __ballot_sync(MHPC_FULL, rlen > 0);
        const int nr = __popc(br);
        if (rlen > 0) {
            const int slot = __popc(br & lt);
            RF[slot] = rf;
            RE[slot] = rincl;
        }
        __syncwarp();
        for (int c = lane; c < ncand; c += 32) {
            int lo = 0, hr = nr - 1;
            while (lo < hr) {
                const int mid = (lo + hr) >> 1;
                if (RE[mid] > c) hr = mid;
                else lo = mid + 1;
            }
            visit(RF[lo] + c - (lo ? RE[lo - 1] : 0));
        }
        __syncwarp();
    }
}

