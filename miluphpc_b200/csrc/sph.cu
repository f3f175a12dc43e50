// SPH: fixed-radius neighbour search, variable smoothing length, density /
// sound speed / pressure, and internal (hydro) forces.
//
// Neighbour search: the reference walks the tree once per particle with a
// per-thread stack (SPH::fixedRadiusNN, src/sph/sph.cu:93-281).  Here a warp
// walks once for 32 consecutive SFC-sorted particles, lane-parallel over a
// shared-memory stack, stages the particles of overlapping leaves and small
// cells as candidates, keeps those that can reach one of the warp's four
// 8-particle sub-groups, and tests each sub-group's particles only against
// its own candidates with the reference's pair rule d^2 < h_i^2 && d^2 < h_j^2
// (j != i), d^2 formed without FMA contraction like the reference build.  All
// pruning is conservative, so the neighbour set equals the brute-force set.
#include "sph.cuh"
#include "walk.cuh"

namespace {

constexpr int kBlock = 128;
constexpr int kWarps = kBlock / 32;
constexpr int kSmall = 16;    // cells with at most this many particles are staged whole

// ------------------------------------------------------------ kernels W
// SmoothingKernel::{spiky, cubicSpline, wendlandc2, wendlandc4, wendlandc6}
// (src/sph/kernel.cu:14-183), 3-D forms, support radius = h.
__device__ __forceinline__ void skernel(int type, double r, double h, double& W, double& dWdr) {
    const double q = r / h;
    W = 0.0;
    dWdr = 0.0;
    switch (type) {
        case 0: {  // spiky
            if (q <= 1.0 && q >= 0.0) {
                const double a = 1.0 - q;
                W = 15. / (M_PI * h * h * h) * a * a * a;
                dWdr = -45 / (M_PI * h * h * h * h) * a * a;
            }
        } break;
        case 1: {  // cubic spline
            const double f = 8. / M_PI * 1. / (h * h * h);
            if (q > 1) {
            } else if (q > 0.5) {
                const double a = 1. - q;
                W = 2. * f * a * a * a;
                dWdr = -6. * f * 1. / h * a * a;
            } else {
                W = f * (6. * q * q * q - 6. * q * q + 1.);
                dWdr = 6. * f / h * (3 * q * q - 2 * q);
            }
        } break;
        case 2: {  // Wendland C2
            if (r <= h) {
                const double a = 1 - q;
                W = 21. / (2 * M_PI * h * h * h) * a * a * a * a * (1 + 4 * q) * (q < 1);
                dWdr = -210. / (M_PI * h * h * h * h) * q * a * a * a * (q < 1);
            }
        } break;
        case 3: {  // Wendland C4 (derivative as written in the reference)
            if (r <= h) {
                const double a = 1 - q, a5 = a * a * a * a * a;
                W = 495. / (32. * M_PI * h * h * h) * a5 * a * (1. + 6. * q + 35. / 3. * q * q) * (q < 1);
                dWdr = -1485. / (16. * M_PI * h * h * h * h) * a5 * (1. - 35. * q * q + 105. * q * q * q) * (q < 1);
            }
        } break;
        default: {  // Wendland C6
            if (r <= h) {
                const double a = 1 - q, a7 = a * a * a * a * a * a * a;
                W = 1365. / (64. * M_PI * h * h * h) * a7 * a * (1. + 8. * q + 25. * q * q + 32 * q * q * q) * (q < 1);
                dWdr = -15015. / (32. * M_PI * h * h * h * h) * q * a7 * (1. + 7 * q + 16 * q * q) * (q < 1);
            }
        } break;
    }
}

// FP32 forms of the same kernels for the mixed-precision pair sums (one
// reciprocal of h, the rest products).
__device__ __forceinline__ void skernel_f(int type, float r, float h, float& W, float& dWdr) {
    const float ih = __frcp_rn(h);
    const float q = r * ih, ih3 = ih * ih * ih, ih4 = ih3 * ih;
    constexpr float kPi = 3.14159265358979f;
    W = 0.f;
    dWdr = 0.f;
    switch (type) {
        case 0: {
            if (q <= 1.f && q >= 0.f) {
                const float a = 1.f - q;
                W = 15.f / kPi * ih3 * a * a * a;
                dWdr = -45.f / kPi * ih4 * a * a;
            }
        } break;
        case 1: {
            const float f = 8.f / kPi * ih3;
            if (q > 1.f) {
            } else if (q > 0.5f) {
                const float a = 1.f - q;
                W = 2.f * f * a * a * a;
                dWdr = -6.f * f * ih * a * a;
            } else {
                W = f * (6.f * q * q * q - 6.f * q * q + 1.f);
                dWdr = 6.f * f * ih * (3.f * q * q - 2.f * q);
            }
        } break;
        case 2: {
            if (q < 1.f) {
                const float a = 1.f - q;
                W = 21.f / (2.f * kPi) * ih3 * a * a * a * a * (1.f + 4.f * q);
                dWdr = -210.f / kPi * ih4 * q * a * a * a;
            }
        } break;
        case 3: {
            if (q < 1.f) {
                const float a = 1.f - q, a5 = a * a * a * a * a;
                W = 495.f / (32.f * kPi) * ih3 * a5 * a * (1.f + 6.f * q + 35.f / 3.f * q * q);
                dWdr = -1485.f / (16.f * kPi) * ih4 * a5 * (1.f - 35.f * q * q + 105.f * q * q * q);
            }
        } break;
        default: {
            if (q < 1.f) {
                const float a = 1.f - q, a7 = a * a * a * a * a * a * a;
                W = 1365.f / (64.f * kPi) * ih3 * a7 * a * (1.f + 8.f * q + 25.f * q * q + 32.f * q * q * q);
                dWdr = -15015.f / (32.f * kPi) * ih4 * q * a7 * (1.f + 7.f * q + 16.f * q * q);
            }
        } break;
    }
}

// FP32 difference of two positions held as FP32 hi/lo splits of FP64 values
__device__ __forceinline__ float3 rel_f(const float4& ah, const float4& al, const float4& bh, const float4& bl) {
    return make_float3((ah.x - bh.x) + (al.x - bl.x), (ah.y - bh.y) + (al.y - bl.y), (ah.z - bh.z) + (al.z - bl.z));
}

// ------------------------------------------------------------ FRNN walk
// One warp per 32 consecutive (sorted or listed) particles, lane = particle,
// four sub-groups of 8 lanes.
//
// Traversal: lane-parallel over a per-warp stack in shared memory.  Every
// step pops up to 32 nodes, one per lane; a node whose particle box misses
// the group's search box (union of [x - h, x + h]), or whose box grown by
// its largest h misses the group's points box, is dropped; leaves, cells of
// at most kSmall particles and shared-key buckets become candidate ranges;
// other cells push their children.  Stack bound as in the gravity list walk:
// a pop of k nodes pushes at most 8k, and k is limited so that a depth-first
// descent (7 per level, 22 levels) always fits on top of the stack.
//
// Candidates: the ranges are expanded 32 at a time; each candidate particle
// is tested against the four sub-groups' boxes (search box, and points box
// grown by h_j when smoothing lengths differ), both rounded outward to FP32
// like the node boxes, so no pair that passes the exact test is dropped.
// Candidates reaching some sub-group go to a shared-memory pool (x, y, z,
// h_j^2, j) and to that sub-group's list.  A full pool is flushed: for each
// sub-group, lane (8q + p) tests particle p of the sub-group against list
// entry 4c + q, so the warp tests 32 pairs per step, and hits are written in
// list order (ballot prefix over the 4 lanes of a particle).
//
// The pair rule is the reference's, d^2 < h_i^2 && d^2 < h_j^2 (j != i), d^2
// formed without FMA contraction; the walk and the box tests are
// conservative, so each neighbour set equals the brute-force set.
//
// mode 0: write lists (h_i = h[i], h_j = h[j]) for all particles; mode 1:
// count only, with h_i = h[i], h_j = h[j] (the variable-h sweep passes the
// sweep's snapshot as h), for the particles of `list` (list_count entries, in
// sorted order, so 32 consecutive entries are still spatially close); mode 2:
// mode 0 for the variable-h iteration on lists: runs only when *gate is
// nonzero, and a count above maxnb (the list keeps its first maxnb entries,
// noi the full count) sets *trunc instead of an error; no statistics.
constexpr int kStack = 512;
constexpr int kReserve = 7 * 22 + 8;
constexpr int kPool = 128;

struct FrnnSmem {
    int stk[kStack];
    double cx[kPool], cy[kPool], cz[kPool], ch2[kPool];  // candidate position, h_j^2
    int cj[kPool];                                        // candidate particle
    unsigned char lst[4][kPool];                          // pool slots per sub-group
    int rf[32], rend[32];                                 // staged ranges: first, end (prefix)
    float4 slo[4], shi[4];                                // sub-group search boxes
    float4 plo[4], phi[4];                                // sub-group points boxes
};

#ifndef MHPC_FRNN_MIN_BLOCKS
#define MHPC_FRNN_MIN_BLOCKS 6
#endif
template <int MODE>
// 6 blocks per SM (the register cap costs a few spilled values, the extra
// warps hide more of the walk's latency)
__global__ void __launch_bounds__(kBlock, MHPC_FRNN_MIN_BLOCKS) k_frnn(TreeDev T, int n, int maxnb, const double* __restrict__ sx,
                                                 const double* __restrict__ sy, const double* __restrict__ sz,
                                                 const double* __restrict__ sh, const int* __restrict__ list,
                                                 const int* __restrict__ list_count,
                                                 const float* __restrict__ node_hmax, int* __restrict__ nbr,
                                                 int* __restrict__ noi, DevStatus* st,
                                                 const int* __restrict__ gate = nullptr, int* trunc = nullptr) {
    __shared__ FrnnSmem smem[kWarps];
    if (st->code) return;
    if (MODE == 2 && *gate == 0) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long g = ((long)blockIdx.x * kBlock + threadIdx.x) >> 5;
    long s = g * 32 + lane;
    bool valid = s < n;
    if (MODE == 1) {
        const long cnt_list = *list_count;
        if (g * 32 >= cnt_list) return;  // whole warp beyond the list
        valid = s < cnt_list;
        s = valid ? list[s] : 0;
    }
    const bool active = valid;
    if (!__any_sync(MHPC_FULL, active)) return;
    FrnnSmem& S = smem[w];
    double px = 0, py = 0, pz = 0, hi = 0;
    if (valid) { px = sx[s]; py = sy[s]; pz = sz[s]; hi = sh[s]; }
    const double hi2 = hi * hi;
    // search box (x +- h) and points box, reduced over the sub-group (8
    // lanes), stored rounded outward, then over the warp
    double lx = active ? px - hi : 1e300, ly = active ? py - hi : 1e300, lz = active ? pz - hi : 1e300;
    double ux = active ? px + hi : -1e300, uy = active ? py + hi : -1e300, uz = active ? pz + hi : -1e300;
    double plx = active ? px : 1e300, ply = active ? py : 1e300, plz = active ? pz : 1e300;
    double pux = active ? px : -1e300, puy = active ? py : -1e300, puz = active ? pz : -1e300;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        lx = fmin(lx, __shfl_xor_sync(MHPC_FULL, lx, o));
        ly = fmin(ly, __shfl_xor_sync(MHPC_FULL, ly, o));
        lz = fmin(lz, __shfl_xor_sync(MHPC_FULL, lz, o));
        ux = fmax(ux, __shfl_xor_sync(MHPC_FULL, ux, o));
        uy = fmax(uy, __shfl_xor_sync(MHPC_FULL, uy, o));
        uz = fmax(uz, __shfl_xor_sync(MHPC_FULL, uz, o));
        plx = fmin(plx, __shfl_xor_sync(MHPC_FULL, plx, o));
        ply = fmin(ply, __shfl_xor_sync(MHPC_FULL, ply, o));
        plz = fmin(plz, __shfl_xor_sync(MHPC_FULL, plz, o));
        pux = fmax(pux, __shfl_xor_sync(MHPC_FULL, pux, o));
        puy = fmax(puy, __shfl_xor_sync(MHPC_FULL, puy, o));
        puz = fmax(puz, __shfl_xor_sync(MHPC_FULL, puz, o));
        if (o == 4 && (lane & 7) == 0) {
            const int q = lane >> 3;
            S.slo[q] = make_float4(__double2float_rd(lx), __double2float_rd(ly), __double2float_rd(lz), 0.f);
            S.shi[q] = make_float4(__double2float_ru(ux), __double2float_ru(uy), __double2float_ru(uz), 0.f);
            S.plo[q] = make_float4(__double2float_rd(plx), __double2float_rd(ply), __double2float_rd(plz), 0.f);
            S.phi[q] = make_float4(__double2float_ru(pux), __double2float_ru(puy), __double2float_ru(puz), 0.f);
        }
    }
    const float qlx = __double2float_rd(lx), qly = __double2float_rd(ly), qlz = __double2float_rd(lz);
    const float qux = __double2float_ru(ux), quy = __double2float_ru(uy), quz = __double2float_ru(uz);
    const float rlx = __double2float_rd(plx), rly = __double2float_rd(ply), rlz = __double2float_rd(plz);
    const float rux = __double2float_ru(pux), ruy = __double2float_ru(puy), ruz = __double2float_ru(puz);
    int k = 0;     // neighbours found for this lane's particle
    int pool = 0;  // pool entries (warp-uniform)
    int cnt0 = 0, cnt1 = 0, cnt2 = 0, cnt3 = 0;  // list entries per sub-group (warp-uniform)
    auto flush = [&]() {
        __syncwarp();
        const int q = lane >> 3, p = lane & 7;
#pragma unroll 1
        for (int sg = 0; sg < 4; ++sg) {
            const int cntg = sg == 0 ? cnt0 : sg == 1 ? cnt1 : sg == 2 ? cnt2 : cnt3;
            const int src = 8 * sg + p;
            const double ix = __shfl_sync(MHPC_FULL, px, src), iy = __shfl_sync(MHPC_FULL, py, src);
            const double iz = __shfl_sync(MHPC_FULL, pz, src), ih2 = __shfl_sync(MHPC_FULL, hi2, src);
            const int is = __shfl_sync(MHPC_FULL, (int)s, src);
            const bool iact = __shfl_sync(MHPC_FULL, (int)active, src) != 0;
            int kb = __shfl_sync(MHPC_FULL, k, src);
            const unsigned pmask = 0x01010101u << p;
            for (int c0 = 0; c0 < cntg; c0 += 4) {
                const int c = c0 + q;
                bool hit = false;
                int j = 0;
                if (iact && c < cntg) {
                    const int slot = S.lst[sg][c];
                    j = S.cj[slot];
                    const double dx = ix - S.cx[slot], dy = iy - S.cy[slot], dz = iz - S.cz[slot];
                    const double d = d2_exact(dx, dy, dz);
                    hit = j != is && d < ih2 && d < S.ch2[slot];
                }
                const unsigned b = __ballot_sync(MHPC_FULL, hit) & pmask;
                if (MODE != 1 && hit) {
                    const int pos = kb + __popc(b & lt);
                    if (pos < maxnb) nbr[nb_index(is, pos, maxnb)] = j;
                }
                kb += __popc(b);
            }
            // lane p (q = 0) holds particle 8 sg + p's count: its owner takes it
            const int knew = __shfl_sync(MHPC_FULL, kb, p);
            if (q == sg) k = knew;
        }
        __syncwarp();
        pool = 0;
        cnt0 = cnt1 = cnt2 = cnt3 = 0;
    };
    // the root's children: node 0 and its skip chain
    int top = 0;
    if (lane == 0) {
        int c = 0;
        while (c < M && top < 8) { S.stk[top++] = c; c = __ldg(&T.link[c].x); }
        if (c < M) set_status(st, MHPC_ERR_DEPTH, 3);
    }
    top = __shfl_sync(MHPC_FULL, top, 0);
    __syncwarp();
    while (top > 0) {
        const int room = (kStack - kReserve - top) / 7;
        int kk = top < 32 ? top : 32;
        if (kk > room) kk = room > 1 ? room : 1;
        const bool act = lane < kk;
        const int nd = act ? S.stk[top - 1 - lane] : 0;
        __syncwarp();
        top -= kk;
        int rf = 0, rlen = 0, kmask = 0;
        if (act) {
            const int2 lk = __ldg(T.link + nd);
            const float4 bl = __ldg(T.bmin + nd), bh = __ldg(T.bmax + nd);
            bool overlap = !(bh.x < qlx || bl.x > qux || bh.y < qly || bl.y > quy || bh.z < qlz || bl.z > quz);
            if (overlap && node_hmax) {
                const float hn = __ldg(node_hmax + nd);
                overlap = !(__fadd_ru(bh.x, hn) < rlx || __fadd_rd(bl.x, -hn) > rux || __fadd_ru(bh.y, hn) < rly ||
                            __fadd_rd(bl.y, -hn) > ruy || __fadd_ru(bh.z, hn) < rlz || __fadd_rd(bl.z, -hn) > ruz);
            }
            if (overlap) {
                rf = __ldg(T.first + nd);
                if (lk.y & ND_LEAF) {
                    rlen = 1;
                } else {
                    const int l = __ldg(T.last + nd);
                    const int km = __ldg(T.kmask + nd);
                    // small cells and shared-key buckets (all particles share
                    // one key) are staged whole; other cells open
                    if (l - rf + 1 <= kSmall || (km & 0x100)) rlen = l - rf + 1;
                    else kmask = km & 0xff;
                }
            }
        }
        // push the children of opened cells
        const int nkid = __popc(kmask);
        int incl = nkid;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(MHPC_FULL, incl, 31);
        if (top + total > kStack) {
            // unreachable by the bound on kk; stop instead of overrunning
            if (lane == 0) set_status(st, MHPC_ERR_DEPTH, 4);
            return;
        }
        if (nkid) {
            const int4 k0 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd));
            const int4 k1 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd) + 1);
            const int all[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
            int wpos = top + incl - nkid;
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((kmask >> d) & 1) S.stk[wpos++] = all[d];
        }
        top += total;
        // staged ranges: compact, with the running end of each
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
            const int r = __popc(br & lt);
            S.rf[r] = rf;
            S.rend[r] = rincl;
        }
        __syncwarp();
        for (int c0 = 0; c0 < ncand; c0 += 32) {
            if (pool + 32 > kPool) flush();
            const int c = c0 + lane;
            int mask = 0, j = 0;
            double qx = 0, qy = 0, qz = 0, hj = 0;
            if (c < ncand) {
                int lo = 0, hi_r = nr - 1;
                while (lo < hi_r) {
                    const int mid = (lo + hi_r) >> 1;
                    if (S.rend[mid] > c) hi_r = mid;
                    else lo = mid + 1;
                }
                j = S.rf[lo] + c - (lo ? S.rend[lo - 1] : 0);
                qx = __ldg(sx + j); qy = __ldg(sy + j); qz = __ldg(sz + j); hj = __ldg(sh + j);
                const float xd = __double2float_rd(qx), xu = __double2float_ru(qx);
                const float yd = __double2float_rd(qy), yu = __double2float_ru(qy);
                const float zd = __double2float_rd(qz), zu = __double2float_ru(qz);
                const float hf = __double2float_ru(hj);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 a = S.slo[q], b = S.shi[q];
                    bool in = !(xu < a.x || xd > b.x || yu < a.y || yd > b.y || zu < a.z || zd > b.z);
                    if (node_hmax) {
                        const float4 e = S.plo[q], f = S.phi[q];
                        in = in && !(__fadd_ru(xu, hf) < e.x || __fadd_rd(xd, -hf) > f.x ||
                                     __fadd_ru(yu, hf) < e.y || __fadd_rd(yd, -hf) > f.y ||
                                     __fadd_ru(zu, hf) < e.z || __fadd_rd(zd, -hf) > f.z);
                    }
                    mask |= (int)in << q;
                }
            }
            const unsigned bp = __ballot_sync(MHPC_FULL, mask != 0);
            if (mask) {
                const int slot = pool + __popc(bp & lt);
                S.cx[slot] = qx; S.cy[slot] = qy; S.cz[slot] = qz; S.ch2[slot] = hj * hj; S.cj[slot] = j;
                const unsigned b0 = __ballot_sync(bp, mask & 1), b1 = __ballot_sync(bp, mask & 2);
                const unsigned b2 = __ballot_sync(bp, mask & 4), b3 = __ballot_sync(bp, mask & 8);
                if (mask & 1) S.lst[0][cnt0 + __popc(b0 & lt)] = (unsigned char)slot;
                if (mask & 2) S.lst[1][cnt1 + __popc(b1 & lt)] = (unsigned char)slot;
                if (mask & 4) S.lst[2][cnt2 + __popc(b2 & lt)] = (unsigned char)slot;
                if (mask & 8) S.lst[3][cnt3 + __popc(b3 & lt)] = (unsigned char)slot;
            }
            const unsigned a0 = __ballot_sync(MHPC_FULL, mask & 1), a1 = __ballot_sync(MHPC_FULL, mask & 2);
            const unsigned a2 = __ballot_sync(MHPC_FULL, mask & 4), a3 = __ballot_sync(MHPC_FULL, mask & 8);
            cnt0 += __popc(a0); cnt1 += __popc(a1); cnt2 += __popc(a2); cnt3 += __popc(a3);
            pool += __popc(bp);
        }
        __syncwarp();
    }
    flush();
    if (active) {
        noi[s] = k;
        if (MODE == 0 && k > maxnb) set_status(st, MHPC_ERR_NEIGHBOURS, (int)s);
        if (MODE == 2 && k > maxnb) *trunc = 1;
        if (MODE == 0) atomicMax(&st->max_noi, k);
    }
    if (MODE == 0) {
        unsigned long long tot = active ? (unsigned long long)k : 0ULL;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(MHPC_FULL, tot, o);
        if (lane == 0) atomicAdd(&st->noi_sum, tot);
    }
}

// Count walk for sparse lists (later variable-h sweeps, where the particles
// still iterating are scattered, so a shared group box would be large): one
// warp per particle (warp_walk), its lanes testing 32 candidates at a time
// with the reference's pair rule.  The longest walks (particles with a large
// h) set a sweep's time, so each particle gets a whole warp.
struct CountVisit {
    const double *sx, *sy, *sz, *sh;
    double px, py, pz, hi2;
    long s;
    int* k;
    __device__ void operator()(int j) const {
        if (j == s) return;
        const double d = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
        const double hj = __ldg(sh + j);
        *k += (d < hi2 && d < hj * hj);
    }
};

__global__ void __launch_bounds__(kBlock) k_count_warp(TreeDev T, const double* __restrict__ sx,
                                                       const double* __restrict__ sy, const double* __restrict__ sz,
                                                       const double* __restrict__ sh, const int* __restrict__ list,
                                                       const int* __restrict__ list_count,
                                                       const float* __restrict__ node_hmax, int* __restrict__ count,
                                                       DevStatus* st) {
    __shared__ int stk[kWarps][kWalkStack];
    __shared__ int rfs[kWarps][32], rends[kWarps][32];
    if (st->code) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long cnt = *list_count;
    const long nwarps = (long)gridDim.x * kWarps;
    for (long q = ((long)blockIdx.x * kBlock + threadIdx.x) >> 5; q < cnt; q += nwarps) {
        const int s = list[q];
        const double px = sx[s], py = sy[s], pz = sz[s], hi = sh[s];
        int k = 0;
        CountVisit v{sx, sy, sz, sh, px, py, pz, hi * hi, (long)s, &k};
        warp_walk(T, M, true, px, py, pz, hi, node_hmax, stk[w], rfs[w], rends[w], st, v);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(MHPC_FULL, k, o);
        if (lane == 0) count[s] = k;
        __syncwarp();
    }
}

// ------------------------------------------------------- variable h update
// Convergence rule and update of fixedRadiusNN_variableSML
// (src/sph/sph.cu:911-933): stop when nit > max_iter or |n - target| < tol,
// provided n < maxnb; otherwise h *= 0.5 (1 + (target / max(n,1))^(1/3)).
//
// The sweep's counts are complete when this runs, so the new h goes straight
// into the snapshot too (hold), and a larger h raises the largest-h bound of
// the particle's leaf and ancestors (grow-only, stopping at the first ancestor
// already as large; a bound left larger than the subtree's h only prunes less).
__global__ void k_vh_update(const int* __restrict__ list, const int* __restrict__ list_count,
                            const int* __restrict__ count, double* h, double* hold, int* done, int* nit, int target,
                            int tol, int max_iter, int maxnb, float* node_hmax, const int* __restrict__ leaf_node,
                            const int* __restrict__ parent, const long long* __restrict__ ord) {
    const int m = *list_count;
    // h never grows past the edge of the (cubic) bounding box: a particle whose
    // neighbours' h do not reach it (an isolated or ejected particle) would
    // otherwise multiply its h by up to 2.46 per sweep, without bound across
    // steps (the reference has no such bound); at the box edge its search
    // already covers every particle.
    const double hcap = ord_to_dbl(ord[1]) - ord_to_dbl(ord[0]);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int i = list[q];
        const int it = ++nit[i];
        const int c = count[i];
        if ((it > max_iter || abs(c - target) < tol) && c < maxnb) {
            done[i] = 1;
        } else {
            const int cc = c < 1 ? 1 : c;
            const double h0 = h[i];
            const double hn = fmin(h0 * (0.5 * (1.0 + pow((double)target / (double)cc, 1. / 3.))), fmax(hcap, h0));
            h[i] = hn;
            hold[i] = hn;
            if (hn > h0) {
                // positive floats order like their bit patterns
                const int v = __float_as_int(__double2float_ru(hn));
                for (int nd = leaf_node[i]; nd >= 0; nd = parent[nd])
                    if (atomicMax(reinterpret_cast<int*>(node_hmax + nd), v) >= v) break;
            }
        }
    }
}

__global__ void k_flags(int n, const int* __restrict__ done, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flags[i] = done[i] ? 0 : 1;
}

__global__ void k_compact(int n, const int* __restrict__ flags, const int* __restrict__ off, int* list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flags[i]) list[off[i]] = i;
}

// number of particles still iterating after the first sweep (the fallback
// count when the first sweep started from predicted smoothing lengths)
__global__ void k_record_active(const int* __restrict__ list_count, int n, DevStatus* st) {
    st->predictor_fallback = *list_count;
    st->predictor_used = n - *list_count;
}

__global__ void k_record_unconverged(const int* __restrict__ list_count, DevStatus* st) {
    st->sml_unconverged = *list_count;
}

__global__ void k_copy(int n, const double* __restrict__ a, double* b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// The particles of `in` that have not stopped, appended to `out` (order
// irrelevant: every particle's update and pair edits depend on it alone, and
// the appended lists are sorted at the end); *out_count must be zero.
__global__ void k_next_list(const int* __restrict__ in, const int* __restrict__ in_count,
                            const int* __restrict__ done, int* out, int* out_count) {
    const int m = *in_count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int i = in[q];
        if (!done[i]) out[atomicAdd(out_count, 1)] = i;
    }
}

// End of a sweep on lists: every iterating particle takes its new h; the
// lists are re-walked when they are truncated (a count above maxnb) or when
// the sweep's pair changes overflowed the event buffer (nothing was edited).
__global__ void k_vh_commit(const int* __restrict__ list, const int* __restrict__ list_count,
                            const double* __restrict__ hnew, double* h, const int* __restrict__ ctr, int* rewalk) {
    const int m = *list_count;
    if (blockIdx.x == 0 && threadIdx.x == 0) *rewalk = (ctr[1] || ctr[2]) ? 1 : 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int i = list[q];
        h[i] = hnew[i];
    }
}

// Statistics and the capacity check of the list walk, for lists that the
// variable-h iteration kept current instead of a final walk.
__global__ void k_noi_stats(int n, int maxnb, const int* __restrict__ noi, DevStatus* st) {
    int mx = 0;
    unsigned long long tot = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int k = noi[i];
        if (k > maxnb) set_status(st, MHPC_ERR_NEIGHBOURS, i);
        mx = max(mx, k);
        tot += (unsigned long long)k;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(MHPC_FULL, mx, o));
        tot += __shfl_xor_sync(MHPC_FULL, tot, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&st->max_noi, mx);
        atomicAdd(&st->noi_sum, tot);
    }
}

// --------------------------------------------------- density + EOS (fused)
// calculateDensity (src/sph/density.cu:8-72), then calculateSoundSpeed
// (src/sph/soundspeed.cu:38-97) and calculatePressure (src/sph/pressure.cu:5-87)
// in the reference's order: the ideal-gas sound speed uses the pressure of
// the previous call.
__global__ void __launch_bounds__(kBlock) k_density_eos(SphParams P, SphSorted S, const int* __restrict__ nbr,
                                                        const int* __restrict__ noi, const int* __restrict__ perm,
                                                        double* rho_out, double* p_out, double* cs_out,
                                                        DevStatus* st) {
    if (st->code) return;
    const long s = (long)blockIdx.x * kBlock + threadIdx.x;
    if (s >= P.n) return;
    const double xi = S.x[s], yi = S.y[s], zi = S.z[s], hi = S.h[s];
    double rho;
    if (P.integrate_density) {
        rho = S.rho[s];
    } else {
        double W, dWdr;
        skernel(P.kernel, 0.0, hi, W, dWdr);
        rho = S.m[s] * W;
        const int k = min(noi[s], P.maxnb);
        for (int q = 0; q < k; ++q) {
            const int j = nbr[nb_index(s, q, P.maxnb)];
            const double hb = P.avg_h ? 0.5 * (hi + __ldg(S.h + j)) : hi;
            const double dx = xi - __ldg(S.x + j), dy = yi - __ldg(S.y + j), dz = zi - __ldg(S.z + j);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            skernel(P.kernel, r, hb, W, dWdr);
            rho += __ldg(S.m + j) * W;
        }
        if (!(rho > 0.0)) set_status(st, MHPC_ERR_NAN, (int)s);
    }
    const int mid = S.mat ? S.mat[s] : 0;
    const MatDev& M = P.mat[mid];
    double p = S.p[s], cs = S.cs[s];
    switch (M.eos_type) {
        case 0: cs = sqrt(M.K * pow(rho, M.gamma - 1.0)); break;
        case 1: case 3: cs = M.cs_init; break;  // constant: initializeSoundSpeed (soundspeed.cu:4-36)
        case 9: cs = sqrt(M.gamma * p / rho); break;
        case 12: cs = 0.0; break;
        default: break;
    }
    switch (M.eos_type) {
        case 0: p = M.K * pow(rho, M.gamma); break;
        case 1: p = (M.bulk / M.n_exp) * (pow(rho / M.rho0, M.n_exp) - 1.0); break;
        case 3: p = 41255.407 * rho; break;
        case 9: p = (M.gamma - 1) * rho * S.e[s]; break;
        case 12: p = cs * cs * rho; break;
        default: break;
    }
    S.rho[s] = rho;
    S.p[s] = p;
    S.cs[s] = cs;
    const int o = perm[s];
    rho_out[o] = rho;
    p_out[o] = p;
    cs_out[o] = cs;
}

// ------------------------------------------------------------- Balsara
// SPH::Kernel::CalcDivvandCurlv (src/sph/kernel.cu:223-342) and the factor of
// internalForces (src/sph/internal_forces.cu:210-217):
//   div v_i = sum_j m_j / rho_j (v_j - v_i) . grad W,
//   curl v_i = sum_j m_j / rho_i (v_i - v_j) x grad W,
//   f_i = |div v_i| / (|div v_i| + |curl v_i| + 1e-4 c_s,i / h_i),
// grad W at h_i (h_bar only under VARIABLE_SML, as in the reference).
__global__ void __launch_bounds__(kBlock) k_balsara(SphParams P, SphSorted S, const int* __restrict__ nbr,
                                                    const int* __restrict__ noi, DevStatus* st) {
    if (st->code) return;
    const long s = (long)blockIdx.x * kBlock + threadIdx.x;
    if (s >= P.n) return;
    const double xi = S.x[s], yi = S.y[s], zi = S.z[s], hi = S.h[s];
    const double vxi = S.vx[s], vyi = S.vy[s], vzi = S.vz[s], rhoi = S.rho[s];
    double divv = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0;
    const int k = min(noi[s], P.maxnb);
    for (int q = 0; q < k; ++q) {
        const int j = nbr[nb_index(s, q, P.maxnb)];
        const double hb = P.variable_sml ? 0.5 * (hi + __ldg(S.h + j)) : hi;
        const double dx = xi - __ldg(S.x + j), dy = yi - __ldg(S.y + j), dz = zi - __ldg(S.z + j);
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        double W, dWdr;
        skernel(P.kernel, r, hb, W, dWdr);
        const double g = dWdr / r;
        const double gx = g * dx, gy = g * dy, gz = g * dz;
        const double dvx = vxi - __ldg(S.vx + j), dvy = vyi - __ldg(S.vy + j), dvz = vzi - __ldg(S.vz + j);
        const double mj = __ldg(S.m + j);
        divv += mj / __ldg(S.rho + j) * (-dvx * gx - dvy * gy - dvz * gz);
        const double w = mj / rhoi;
        c0 += w * (dvy * gz - dvz * gy);
        c1 += w * (dvz * gx - dvx * gz);
        c2 += w * (dvx * gy - dvy * gx);
    }
    const double curl = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    S.bal[s] = fabs(divv) / (fabs(divv) + curl + 1e-4 * S.cs[s] / hi);
}

// ------------------------------------------------------------- forces
// SPH::Kernel::internalForces, hydro part, SPH_EQU_VERSION 1
// (src/sph/internal_forces.cu:372-552).
__global__ void __launch_bounds__(kBlock) k_forces(SphParams P, SphSorted S, const int* __restrict__ nbr,
                                                   const int* __restrict__ noi, const int* __restrict__ perm,
                                                   double* ax_o, double* ay_o, double* az_o, double* drhodt_o,
                                                   double* dedt_o, double* dsmldt_o, DevStatus* st) {
    if (st->code) return;
    const long s = (long)blockIdx.x * kBlock + threadIdx.x;
    if (s >= P.n) return;
    const double xi = S.x[s], yi = S.y[s], zi = S.z[s], hi = S.h[s];
    const double vxi = S.vx[s], vyi = S.vy[s], vzi = S.vz[s];
    const double rhoi = S.rho[s], pi = S.p[s], csi = S.cs[s];
    const int mid = S.mat ? S.mat[s] : 0;
    const double alpha = P.mat[mid].alpha, beta = P.mat[mid].beta;
    const double pri = pi / (rhoi * rhoi);
    double a0 = 0, a1 = 0, a2 = 0, drho = 0, de = 0, dh = 0;
    const int k = min(noi[s], P.maxnb);
    for (int q = 0; q < k; ++q) {
        const int j = nbr[nb_index(s, q, P.maxnb)];
        const double hj = __ldg(S.h + j);
        const double hb = P.avg_h ? 0.5 * (hi + hj) : hi;
        const double dx = xi - __ldg(S.x + j), dy = yi - __ldg(S.y + j), dz = zi - __ldg(S.z + j);
        const double rr = dx * dx + dy * dy + dz * dz;
        const double r = sqrt(rr);
        double W, dWdr;
        skernel(P.kernel, r, hb, W, dWdr);
        const double g = dWdr / r;
        const double gx = g * dx, gy = g * dy, gz = g * dz;
        const double dvx = vxi - __ldg(S.vx + j), dvy = vyi - __ldg(S.vy + j), dvz = vzi - __ldg(S.vz + j);
        const double vvnablaW = dvx * gx + dvy * gy + dvz * gz;
        const double vr = dvx * dx + dvy * dy + dvz * dz;
        const double rhoj = __ldg(S.rho + j), mj = __ldg(S.m + j);
        double pij = 0.0;
        if (vr < 0) {
            const double csbar = 0.5 * (csi + __ldg(S.cs + j));
            const double smooth = 0.5 * (hi + hj);
            double mu = smooth * vr / (rr + smooth * smooth * 1e-2);
            const double rhobar = 0.5 * (rhoi + rhoj);
            if (P.balsara) mu *= (S.bal[s] + __ldg(S.bal + j)) / 2.;
            pij = (beta * mu - alpha * csbar) * mu / rhobar;
        }
        const double pf = -mj * (pri + __ldg(S.p + j) / (rhoj * rhoj));
        const double ajx = pf * gx, ajy = pf * gy, ajz = pf * gz;
        const double vf = mj * (-pij);
        a0 += ajx + vf * gx;
        a1 += ajy + vf * gy;
        a2 += ajz + vf * gz;
        drho += rhoi / rhoj * mj * vvnablaW;
        if (P.integrate_sml) dh -= 1. / 3. * hi * mj / rhoj * vvnablaW;
        if (P.integrate_energy) de += 0.5 * mj * pij * vvnablaW - 0.5 * (ajx * dvx + ajy * dvy + ajz * dvz);
    }
    const int o = perm[s];
    ax_o[o] = a0;
    ay_o[o] = a1;
    az_o[o] = a2;
    if (drhodt_o) drhodt_o[o] = drho;
    if (dedt_o) dedt_o[o] = P.integrate_energy ? de : 0.0;
    if (dsmldt_o) dsmldt_o[o] = P.integrate_sml ? dh : 0.0;
}

// ----------------------------------------------- mixed precision (FP32 pairs)
// Positions as FP32 hi/lo splits: x_hi = (float)x, x_lo = (float)(x - x_hi), so
// that a neighbour difference (x_hi,i - x_hi,j) + (x_lo,i - x_lo,j) keeps FP32
// relative accuracy of the difference itself at any distance from the origin.
__global__ void k_pack_pos(SphSorted S, int n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const double x = S.x[s], y = S.y[s], z = S.z[s];
        const float hx = (float)x, hy = (float)y, hz = (float)z;
        S.f0[s] = make_float4(hx, hy, hz, (float)S.h[s]);
        S.f1[s] = make_float4((float)(x - (double)hx), (float)(y - (double)hy), (float)(z - (double)hz), (float)S.m[s]);
    }
}

// EOS of one particle (calculateSoundSpeed, then calculatePressure, in the
// reference's order: the ideal-gas sound speed uses the previous pressure)
__device__ __forceinline__ void eos(const MatDev& M, double rho, double e, double& p, double& cs) {
    switch (M.eos_type) {
        case 0: cs = sqrt(M.K * pow(rho, M.gamma - 1.0)); break;
        case 1: case 3: cs = M.cs_init; break;  // constant: initializeSoundSpeed (soundspeed.cu:4-36)
        case 9: cs = sqrt(M.gamma * p / rho); break;
        case 12: cs = 0.0; break;
        default: break;
    }
    switch (M.eos_type) {
        case 0: p = M.K * pow(rho, M.gamma); break;
        case 1: p = (M.bulk / M.n_exp) * (pow(rho / M.rho0, M.n_exp) - 1.0); break;
        case 3: p = 41255.407 * rho; break;
        case 9: p = (M.gamma - 1) * rho * e; break;
        case 12: p = cs * cs * rho; break;
        default: break;
    }
}

__global__ void __launch_bounds__(kBlock) k_density_eos_f32(SphParams P, SphSorted S, const int* __restrict__ nbr,
                                                            const int* __restrict__ noi, const int* __restrict__ perm,
                                                            double* rho_out, double* p_out, double* cs_out,
                                                            DevStatus* st) {
    if (st->code) return;
    const long s = (long)blockIdx.x * kBlock + threadIdx.x;
    if (s >= P.n) return;
    double rho;
    if (P.integrate_density) {
        rho = S.rho[s];
    } else {
        const float4 a0 = S.f0[s], a1 = S.f1[s];
        const float hi = a0.w;
        float W, dWdr;
        skernel_f(P.kernel, 0.f, hi, W, dWdr);
        rho = (double)(a1.w * W);
        const int k = min(noi[s], P.maxnb);
        for (int q = 0; q < k; ++q) {
            const int j = nbr[nb_index(s, q, P.maxnb)];
            const float4 b0 = __ldg(S.f0 + j), b1 = __ldg(S.f1 + j);
            const float3 d = rel_f(a0, a1, b0, b1);
            const float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
            skernel_f(P.kernel, r, P.avg_h ? 0.5f * (hi + b0.w) : hi, W, dWdr);
            rho += (double)(b1.w * W);
        }
        if (!(rho > 0.0)) set_status(st, MHPC_ERR_NAN, (int)s);
    }
    const int mid = S.mat ? S.mat[s] : 0;
    double p = S.p[s], cs = S.cs[s];
    eos(P.mat[mid], rho, S.e[s], p, cs);
    S.rho[s] = rho;
    S.p[s] = p;
    S.cs[s] = cs;
    S.f2[s] = make_float4((float)S.vx[s], (float)S.vy[s], (float)S.vz[s], (float)cs);
    S.f3[s] = make_float2((float)rho, (float)(p / (rho * rho)));
    const int o = perm[s];
    rho_out[o] = rho;
    p_out[o] = p;
    cs_out[o] = cs;
}

__global__ void __launch_bounds__(kBlock) k_forces_f32(SphParams P, SphSorted S, const int* __restrict__ nbr,
                                                       const int* __restrict__ noi, const int* __restrict__ perm,
                                                       double* ax_o, double* ay_o, double* az_o, double* drhodt_o,
                                                       double* dedt_o, double* dsmldt_o, DevStatus* st) {
    if (st->code) return;
    const long s = (long)blockIdx.x * kBlock + threadIdx.x;
    if (s >= P.n) return;
    const float4 a0 = S.f0[s], a1 = S.f1[s], v = S.f2[s];
    const float2 rp = S.f3[s];
    const float hi = a0.w, csi = v.w, rhoi = rp.x, pri = rp.y;
    const int mid = S.mat ? S.mat[s] : 0;
    const float alpha = (float)P.mat[mid].alpha, beta = (float)P.mat[mid].beta;
    const float bali = P.balsara ? (float)S.bal[s] : 1.f;
    double a0x = 0, a0y = 0, a0z = 0, drho = 0, de = 0, dh = 0;
    const int k = min(noi[s], P.maxnb);
    for (int q = 0; q < k; ++q) {
        const int j = nbr[nb_index(s, q, P.maxnb)];
        const float4 b0 = __ldg(S.f0 + j), b1 = __ldg(S.f1 + j), w = __ldg(S.f2 + j);
        const float2 rpj = __ldg(S.f3 + j);
        const float hj = b0.w, mj = b1.w, rhoj = rpj.x;
        const float3 d = rel_f(a0, a1, b0, b1);
        const float rr = d.x * d.x + d.y * d.y + d.z * d.z;
        const float r = sqrtf(rr);
        float W, dWdr;
        skernel_f(P.kernel, r, P.avg_h ? 0.5f * (hi + hj) : hi, W, dWdr);
        const float g = __fdividef(dWdr, r);
        const float gx = g * d.x, gy = g * d.y, gz = g * d.z;
        const float dvx = v.x - w.x, dvy = v.y - w.y, dvz = v.z - w.z;
        const float vvnablaW = dvx * gx + dvy * gy + dvz * gz;
        const float vr = dvx * d.x + dvy * d.y + dvz * d.z;
        float pij = 0.f;
        if (vr < 0.f) {
            const float csbar = 0.5f * (csi + w.w);
            const float smooth = 0.5f * (hi + hj);
            float mu = __fdividef(smooth * vr, rr + smooth * smooth * 1e-2f);
            if (P.balsara) mu *= 0.5f * (bali + (float)__ldg(S.bal + j));
            pij = __fdividef((beta * mu - alpha * csbar) * mu, 0.5f * (rhoi + rhoj));
        }
        const float pf = -mj * (pri + rpj.y);
        const float ajx = pf * gx, ajy = pf * gy, ajz = pf * gz;
        const float vf = -mj * pij;
        a0x += (double)(ajx + vf * gx);
        a0y += (double)(ajy + vf * gy);
        a0z += (double)(ajz + vf * gz);
        const float mv = __fdividef(mj, rhoj) * vvnablaW;
        drho += (double)(rhoi * mv);
        if (P.integrate_sml) dh -= (double)(1.f / 3.f * hi * mv);
        if (P.integrate_energy) de += (double)(0.5f * mj * pij * vvnablaW - 0.5f * (ajx * dvx + ajy * dvy + ajz * dvz));
    }
    const int o = perm[s];
    ax_o[o] = a0x;
    ay_o[o] = a0y;
    az_o[o] = a0z;
    if (drhodt_o) drhodt_o[o] = drho;
    if (dedt_o) dedt_o[o] = P.integrate_energy ? de : 0.0;
    if (dsmldt_o) dsmldt_o[o] = P.integrate_sml ? dh : 0.0;
}

__global__ void k_export_nnl(int n, int maxnb, const int* __restrict__ nbr, const int* __restrict__ noi,
                             const int* __restrict__ perm, int* nnl, int* noi_out) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = perm[s];
        const int k = noi[s];
        if (noi_out) noi_out[o] = k;
        if (nnl) {
            const int kk = min(k, maxnb);
            for (int q = 0; q < maxnb; ++q)
                nnl[(size_t)o * maxnb + q] = q < kk ? perm[nbr[nb_index(s, q, maxnb)]] : -1;
        }
    }
}

}  // namespace

int sph_frnn(const TreeDev& T, const SphParams& P, const SphSorted& S, int* nbr, int* noi, DevStatus* st,
             cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    long blocks = (((long)P.n + 31) / 32 * 32 + kBlock - 1) / kBlock;
    const float* hmax = nullptr;
    if (P.avg_h) {  // smoothing lengths differ: prune nodes by their largest h
        int rc = tree_node_hmax(T, S.h, st, s);
        if (rc) return rc;
        hmax = T.hmax;
    }
    k_frnn<0><<<(int)blocks, kBlock, 0, s>>>(T, P.n, P.maxnb, S.x, S.y, S.z, S.h, nullptr, nullptr, hmax, nbr, noi,
                                              st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_variable_h(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                   double* h, const VhBuffers& B, int target, int tol, int max_iter, int sweeps, DevStatus* st,
                   cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    const long blocks = (((long)P.n + 31) / 32 * 32 + kBlock - 1) / kBlock;
    const int g = grid_for(P.n, 256, 148 * 16);
    const int* list_count = B.off + P.n;
    // Jacobi snapshot of h and the largest-h bounds; k_vh_update keeps both
    // current from then on
    k_copy<<<g, 256, 0, s>>>(P.n, h, B.hold);
    int rc0 = tree_node_hmax(T, B.hold, st, s);
    if (rc0) return rc0;
    for (int it = 0; it < sweeps; ++it) {
        // the list of particles still iterating
        k_flags<<<g, 256, 0, s>>>(P.n, B.done, B.flags);
        int rc = scan_exclusive_i32(B.flags, B.off, P.n, B.scan_scratch, s);
        if (rc) return rc;
        k_compact<<<g, 256, 0, s>>>(P.n, B.flags, B.off, B.list);
        if (it == 1) k_record_active<<<1, 1, 0, s>>>(list_count, P.n, st);
        if (it == 0) {
            // first sweep: (nearly) every particle, group walks
            k_frnn<1><<<(int)blocks, kBlock, 0, s>>>(T, P.n, P.maxnb, x, y, z, B.hold, B.list, list_count, T.hmax,
                                                      nullptr, B.count, st);
        } else {
            // later sweeps: the few particles still iterating, a warp each
            k_count_warp<<<148 * 8, kBlock, 0, s>>>(T, x, y, z, B.hold, B.list, list_count, T.hmax, B.count, st);
        }
        k_vh_update<<<g, 256, 0, s>>>(B.list, list_count, B.count, h, B.hold, B.done, B.nit, target, tol, max_iter,
                                      P.maxnb, T.hmax, T.leaf_node, T.parent, P.ord);
    }
    k_flags<<<g, 256, 0, s>>>(P.n, B.done, B.flags);
    int rc = scan_exclusive_i32(B.flags, B.off, P.n, B.scan_scratch, s);
    if (rc) return rc;
    k_record_unconverged<<<1, 1, 0, s>>>(list_count, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_variable_h_lists(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                         double* h, int* nbr, int* noi, const VhBuffers& V, const BandBuffers& B, int target,
                         int tol, int max_iter, int sweeps, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    const long blocks = (((long)P.n + 31) / 32 * 32 + kBlock - 1) / kBlock;
    const int g = grid_for(P.n, 256, 148 * 16);
    const int* list_count = V.off + P.n;
    int* trunc = B.ctr + 2;   // some list holds fewer entries than its count
    int* rewalk = B.ctr + 3;  // the lists are re-walked after this sweep
    double* hnew = B.hnew;
    CUDA_TRY(cudaMemsetAsync(B.ctr, 0, sizeof(int) * 4, s));
    CUDA_TRY(cudaMemsetAsync(rewalk, 1, sizeof(int), s));  // nonzero: the first walk runs
    CUDA_TRY(cudaMemsetAsync(B.dirty, 0, sizeof(int) * P.n, s));
    k_copy<<<g, 256, 0, s>>>(P.n, h, hnew);
    int rc = tree_node_hmax(T, h, st, s);
    if (rc) return rc;
    // the lists and counts of the starting h: the counts of the first sweep
    k_frnn<2><<<(int)blocks, kBlock, 0, s>>>(T, P.n, P.maxnb, x, y, z, h, nullptr, nullptr, T.hmax, nbr, noi, st,
                                              rewalk, trunc);
    // the first sweep lists every particle (ordered, by a scan); later sweeps
    // keep the particles of the previous list that have not stopped
    k_flags<<<g, 256, 0, s>>>(P.n, V.done, V.flags);
    rc = scan_exclusive_i32(V.flags, V.off, P.n, V.scan_scratch, s);
    if (rc) return rc;
    k_compact<<<g, 256, 0, s>>>(P.n, V.flags, V.off, V.list);
    const int* cur = V.list;
    const int* cur_count = list_count;
    for (int it = 0; it < sweeps; ++it) {
        if (it > 0) {
            int* out = (it & 1) ? V.list2 : V.list;
            int* out_count = V.cnt + (it & 1);
            CUDA_TRY(cudaMemsetAsync(out_count, 0, sizeof(int), s));
            k_next_list<<<g, 256, 0, s>>>(cur, cur_count, V.done, out, out_count);
            cur = out;
            cur_count = out_count;
        }
        if (it == 1) k_record_active<<<1, 1, 0, s>>>(cur_count, P.n, st);
        // the reference's update from the exact counts of the current h (Jacobi:
        // every new h goes to hnew first)
        k_vh_update<<<g, 256, 0, s>>>(cur, cur_count, noi, hnew, hnew, V.done, V.nit, target, tol, max_iter,
                                      P.maxnb, T.hmax, T.leaf_node, T.parent, P.ord);
        rc = sph_apply_h_changes(T, P, x, y, z, h, hnew, nbr, noi, cur, cur_count, B, trunc, st, s);
        if (rc) return rc;
        k_vh_commit<<<g, 256, 0, s>>>(cur, cur_count, hnew, h, B.ctr, rewalk);
        k_frnn<2><<<(int)blocks, kBlock, 0, s>>>(T, P.n, P.maxnb, x, y, z, h, nullptr, nullptr, T.hmax, nbr, noi,
                                                  st, rewalk, trunc);
    }
    {
        int* out = (sweeps & 1) ? V.list2 : V.list;
        int* out_count = V.cnt + (sweeps & 1);
        CUDA_TRY(cudaMemsetAsync(out_count, 0, sizeof(int), s));
        k_next_list<<<g, 256, 0, s>>>(cur, cur_count, V.done, out, out_count);
        k_record_unconverged<<<1, 1, 0, s>>>(out_count, st);
    }
    rc = sph_sort_appended(P, nbr, noi, B.appended, s);
    if (rc) return rc;
    k_noi_stats<<<g, 256, 0, s>>>(P.n, P.maxnb, noi, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_density_eos(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, const int* perm,
                    double* rho_out, double* p_out, double* cs_out, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    if (P.mixed) {
        if (!S.f0 || !S.f1 || !S.f2 || !S.f3) return MHPC_ERR_ARG;
        k_pack_pos<<<grid_for(P.n, 256, 148 * 8), 256, 0, s>>>(S, P.n);
        k_density_eos_f32<<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, S, nbr, noi, perm, rho_out, p_out,
                                                                        cs_out, st);
        CUDA_TRY(cudaGetLastError());
        return MHPC_OK;
    }
    k_density_eos<<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, S, nbr, noi, perm, rho_out, p_out, cs_out, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_balsara(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, DevStatus* st,
                cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    k_balsara<<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, S, nbr, noi, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_forces(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, const int* perm, double* ax,
               double* ay, double* az, double* drhodt, double* dedt, double* dsmldt, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    if (P.mixed) {
        if (!S.f0 || !S.f1 || !S.f2 || !S.f3) return MHPC_ERR_ARG;
        k_forces_f32<<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, S, nbr, noi, perm, ax, ay, az, drhodt, dedt,
                                                                   dsmldt, st);
        CUDA_TRY(cudaGetLastError());
        return MHPC_OK;
    }
    k_forces<<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, S, nbr, noi, perm, ax, ay, az, drhodt, dedt, dsmldt,
                                                           st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

namespace {
__global__ void k_band(int n, const int* __restrict__ noi, int target, int tol, DevStatus* st) {
    int bad = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        bad += abs(noi[i] - target) >= tol;
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(MHPC_FULL, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&st->sml_out_of_band, bad);
}
}  // namespace

int sph_band_stats(const SphParams& P, const int* noi, int target, int tol, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    k_band<<<grid_for(P.n, 256, 148 * 4), 256, 0, s>>>(P.n, noi, target, tol, st);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_export_nnl(const SphParams& P, const int* nbr, const int* noi, const int* perm, int* nnl, int* noi_out,
                   cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    k_export_nnl<<<grid_for(P.n, 256, 148 * 16), 256, 0, s>>>(P.n, P.maxnb, nbr, noi, perm, nnl, noi_out);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
