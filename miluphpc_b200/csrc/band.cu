// Neighbour-band repair: the rule is stated next to sph_band_fixup in sph.cuh.
//
// The variable-h iteration of the reference (fixedRadiusNN_variableSML,
// src/sph/sph.cu:739-961) stops a particle once its count is inside
// |n - target| < tol (sph.cu:911-933), but the count of a particle that has
// stopped keeps moving while its neighbours' h change (a pair counts when
// d < min(h_i, h_j)), and a particle that reaches the iteration limit stops
// wherever it is.  After the list walk every count is exact, so each round
// here starts from the lists: the particles out of the band pick a new h by
// selection among their candidates (all other h frozen), and the pairs whose
// status changes are removed from or appended to both lists.
//
// Kernels of one round: flags + scan + compaction (out-of-band list),
// k_band_select (selection, 8 lanes per particle: a tree walk below the band,
// the particle's own list above it), k_band_events (one event per changed
// pair, likewise), k_band_remove (tombstones),
// k_band_compact, k_band_add, k_band_commit.  Every kernel after the
// compaction reads the list length on the device and returns at once when it
// is zero, so the host enqueues all rounds without synchronising.
#include "sph.cuh"

namespace {

constexpr int kBandBlock = 64;  // 2 warps, 8 particles (8 lanes each)
constexpr int kBandWarps = kBandBlock / 32;
constexpr int kBandCap = 256;   // candidates held per particle during the selection
constexpr int kBandStack = 256;
constexpr int kBandReserve = 7 * 22 + 8;
constexpr int kBandSmall = 16;  // cells with at most this many particles are tested whole

// One particle per 8-lane segment of the warp (all 32 lanes call this).
// Visits every particle j of the leaves, small cells and shared-key buckets
// whose box comes within `rad` of the particle and whose largest h below the
// node reaches it: visit(j) is called on one lane of the segment per
// candidate (j may be the particle itself).  Pruning is conservative (FP32
// boxes rounded outward), so every j with d < rad and d < h_j is visited.
// Stack bound as in the other walks: a pop of k nodes pushes at most 8k.
template <class Visit>
__device__ void band_walk(const TreeDev& T, int M, bool valid, double px, double py, double pz, double rad,
                          const float* __restrict__ node_hmax, int* S, int* RF, int* RE, DevStatus* st,
                          Visit& visit) {
    const int lane = threadIdx.x & 31, sg = lane >> 3, r = lane & 7;
    const unsigned seg = 0xffu << (8 * sg);
    const unsigned lt = (1u << lane) - 1u;
    const float lx = __double2float_rd(px - rad), ly = __double2float_rd(py - rad), lz = __double2float_rd(pz - rad);
    const float ux = __double2float_ru(px + rad), uy = __double2float_ru(py + rad), uz = __double2float_ru(pz + rad);
    const float fx0 = __double2float_rd(px), fy0 = __double2float_rd(py), fz0 = __double2float_rd(pz);
    const float fx1 = __double2float_ru(px), fy1 = __double2float_ru(py), fz1 = __double2float_ru(pz);
    int top = 0;
    if (valid && r == 0) {
        int c = 0;
        while (c < M && top < 8) { S[top++] = c; c = __ldg(&T.link[c].x); }
        if (c < M) set_status(st, MHPC_ERR_DEPTH, 7);
    }
    top = __shfl_sync(MHPC_FULL, top, lane & ~7);
    __syncwarp();
    while (__any_sync(MHPC_FULL, top > 0)) {
        const int room = (kBandStack - kBandReserve - top) / 7;
        int kk = top < 8 ? top : 8;
        if (kk > room) kk = room > 1 ? room : 1;
        if (top == 0) kk = 0;
        const bool act = r < kk;
        const int nd = act ? S[top - 1 - r] : 0;
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
                    if (l - rf + 1 <= kBandSmall || (km & 0x100)) rlen = l - rf + 1;
                    else kmask = km & 0xff;
                }
            }
        }
        const int nkid = __popc(kmask);
        int incl = nkid;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, incl, o, 8);
            if (r >= o) incl += v;
        }
        const int total = __shfl_sync(MHPC_FULL, incl, 7, 8);
        const bool over = top + total > kBandStack;  // unreachable by the bound on kk
        if (over && r == 0 && valid) set_status(st, MHPC_ERR_DEPTH, 8);
        if (nkid && !over) {
            const int4 k0 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd));
            const int4 k1 = __ldg(reinterpret_cast<const int4*>(T.kids + 8 * (size_t)nd) + 1);
            const int all[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
            int wpos = top + incl - nkid;
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if ((kmask >> d) & 1) S[wpos++] = all[d];
        }
        top = over ? 0 : top + total;
        int rincl = rlen;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int v = __shfl_up_sync(MHPC_FULL, rincl, o, 8);
            if (r >= o) rincl += v;
        }
        const int ncand = __shfl_sync(MHPC_FULL, rincl, 7, 8);
        const unsigned br = __ballot_sync(MHPC_FULL, rlen > 0) & seg;
        const int nr = __popc(br);
        if (rlen > 0) {
            const int slot = __popc(br & lt);
            RF[slot] = rf;
            RE[slot] = rincl;
        }
        __syncwarp();
        int maxc = ncand;
        maxc = max(maxc, __shfl_xor_sync(MHPC_FULL, maxc, 8));
        maxc = max(maxc, __shfl_xor_sync(MHPC_FULL, maxc, 16));
        for (int c0 = 0; c0 < maxc; c0 += 8) {
            const int c = c0 + r;
            if (c < ncand) {
                int lo = 0, hr = nr - 1;
                while (lo < hr) {
                    const int mid = (lo + hr) >> 1;
                    if (RE[mid] > c) hr = mid;
                    else lo = mid + 1;
                }
                visit(RF[lo] + c - (lo ? RE[lo - 1] : 0));
            }
        }
        __syncwarp();
    }
}

// The band's two repair targets and the search radius of a particle with
// count n and smoothing length h (the same arithmetic as the oracle's).
struct BandRule {
    int target, tol;
    __device__ bool out(int n) const { return abs(n - target) >= tol; }
    __device__ int want(int n) const { return n >= target + tol ? target + tol - 2 : target - tol + 2; }
    __device__ double radius(int n, double h) const {
        if (n >= target + tol) return h;
        return 2 * n >= want(n) ? 1.5 * h : 2.0 * h;
    }
};

struct SelectSmem {
    int stk[kBandStack];
    int rf[8], re[8];
    double d2[kBandCap];
    int cnt;
};

struct SelectVisit {
    const double *sx, *sy, *sz, *h;
    double px, py, pz, rad2;
    long s;
    SelectSmem* m;
    __device__ void operator()(int j) const {
        if (j == s) return;
        const double d2 = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
        const double hj = __ldg(h + j);
        if (d2 < rad2 && d2 < hj * hj) {
            const int k = atomicAdd(&m->cnt, 1);
            if (k < kBandCap) m->d2[k] = d2;
        }
    }
};

// Out-of-band list of this round; in round 0 its length is recorded as the
// count before any repair.
__global__ void k_band_flags(int n, const int* __restrict__ noi, BandRule R, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flags[i] = R.out(noi[i]) ? 1 : 0;
}

__global__ void k_band_compact_list(int n, const int* __restrict__ flags, const int* __restrict__ off, int* list,
                                    int* ctr, DevStatus* st, int round) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flags[i]) list[off[i]] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctr[0] = 0;  // events
        ctr[1] = 0;  // overflow
        if (round == 0) st->sml_band_before = off[n];
    }
}

// Selection: candidates of particle i within its search radius; on more than
// kBandCap candidates the radius shrinks by 0.8 (at most 4 times; the wanted
// rank still lies inside while more than `want` candidates remain), then:
// more than `want` candidates -> the midpoint of the want-th and
// (want+1)-th smallest distances; otherwise the radius itself; still too many
// -> h unchanged.  A particle above the band searches within its own h, so
// its candidates are exactly its neighbour list (d < h_i and d < h_j): it
// reads them from the list instead of walking the tree.  A new h above the
// old one raises the largest-h bounds of the particle's leaf and ancestors
// (grow-only).
__global__ void __launch_bounds__(kBandBlock) k_band_select(TreeDev T, const double* __restrict__ sx,
                                                            const double* __restrict__ sy,
                                                            const double* __restrict__ sz,
                                                            const double* __restrict__ h,
                                                            const double* __restrict__ h0,
                                                            const int* __restrict__ noi,
                                                            const int* __restrict__ nbr, int maxnb,
                                                            const int* __restrict__ list,
                                                            const int* __restrict__ list_count, BandRule R,
                                                            double* hnew, float* node_hmax, DevStatus* st) {
    __shared__ SelectSmem smem[kBandWarps][4];
    if (st->code) return;
    const long cnt = *list_count;
    if (cnt == 0) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sg = lane >> 3, r = lane & 7;
    SelectSmem* m = &smem[w][sg];
    const long nwarps = (long)gridDim.x * kBandWarps;
    for (long gw = ((long)blockIdx.x * kBandBlock + threadIdx.x) >> 5; gw * 4 < cnt; gw += nwarps) {
        const long q = gw * 4 + sg;
        const bool valid = q < cnt;
        const int s = valid ? list[q] : 0;
        const double px = sx[s], py = sy[s], pz = sz[s], hi = h[s];
        const int ni = noi[s];
        const int want = R.want(ni);
        const bool above = ni >= R.target + R.tol;
        // from below at most twice the h before the first round (at a free
        // surface the neighbours' h may not reach the particle at all)
        double rad = above ? R.radius(ni, hi) : fmin(R.radius(ni, hi), 2.0 * h0[s]);
        // the list holds the candidates of a particle above the band
        const bool from_list = valid && above && ni <= min(maxnb, kBandCap);
        bool done = !valid;
        double result = hi;
        for (int attempt = 0; attempt < 5; ++attempt) {
            if (r == 0) m->cnt = from_list ? ni : 0;
            __syncwarp();
            if (from_list) {
                for (int k = r; k < ni; k += 8) {
                    const int j = nbr[nb_index(s, k, maxnb)];
                    m->d2[k] = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
                }
            }
            SelectVisit v{sx, sy, sz, h, px, py, pz, rad * rad, (long)s, m};
            // a finished segment, or one reading its list, walks nothing
            const bool walk = valid && !done && !from_list;
            band_walk(T, M, walk, px, py, pz, walk ? rad : -1.0, node_hmax, m->stk, m->rf, m->re, st, v);
            __syncwarp();
            const int found = m->cnt;
            const bool in_cap = !done && found <= kBandCap;
            const bool pick = in_cap && found > want;
            // ranks by counting (d2 ascending; equal distances have equal values,
            // so the two order statistics do not depend on how ties are broken)
            double lo = -1.0, hi2 = -1.0;
            if (pick) {
                for (int a = r; a < found; a += 8) {
                    const double da = m->d2[a];
                    int rank = 0;
                    for (int b = 0; b < found; ++b) {
                        const double db = m->d2[b];
                        rank += (db < da) || (db == da && b < a);
                    }
                    if (rank == want - 1) lo = da;
                    if (rank == want) hi2 = da;
                }
            }
            // every lane takes part; width 8 keeps each exchange inside its segment
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                lo = fmax(lo, __shfl_xor_sync(MHPC_FULL, lo, o, 8));
                hi2 = fmax(hi2, __shfl_xor_sync(MHPC_FULL, hi2, o, 8));
            }
            if (in_cap) {
                result = pick ? 0.5 * (sqrt(lo) + sqrt(hi2)) : rad;
                done = true;
            } else if (!done) {
                rad = 0.8 * rad;
            }
            __syncwarp();
            if (__all_sync(MHPC_FULL, done)) break;
        }
        // still more than kBandCap candidates after the last shrink: unchanged
        if (valid && r == 0) {
            hnew[s] = result;
            if (result > hi) {
                const int vbits = __float_as_int(__double2float_ru(result));
                for (int nd = T.leaf_node[s]; nd >= 0; nd = T.parent[nd])
                    if (atomicMax(reinterpret_cast<int*>(node_hmax + nd), vbits) >= vbits) break;
            }
        }
        __syncwarp();
    }
}

struct EventSmem {
    int stk[kBandStack];
    int rf[8], re[8];
};

// Who reports a pair whose status changes.  A particle above the band only
// lowers its h, so it only loses pairs, all of them in its list; a particle
// below only raises it and walks the tree for the pairs it gains or loses.
// A pair is reported by its out-of-band end if it has one; of two ends out of
// the band on the same side, by the smaller index; of one above and one
// below, by the one below (the walk sees every pair the list can miss).
__device__ __forceinline__ bool reports(const BandRule& R, bool i_below, long i, int j, int nj) {
    if (!R.out(nj)) return true;
    const bool j_below = nj < R.target;
    if (i_below != j_below) return i_below;
    return i < j;
}

// Pair changes of a particle below the band: every j within max(h_i, h_i')
// with d < max(h_j, h_j'); the pair is present before when d < min(h_i, h_j)
// and after when d < min(h_i', h_j') (the list walk's test, d^2 against h^2).
struct EventVisit {
    const double *sx, *sy, *sz, *h, *hn;
    const int* noi;
    BandRule R;
    double px, py, pz, hio2, hin2;
    long s;
    int2* ev;
    int cap;
    int* ctr;
    __device__ void operator()(int j) const {
        if (j == s) return;
        const double d2 = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
        const double hjo = h[j], hjn = hn[j];
        const bool was = d2 < hio2 && d2 < hjo * hjo;
        const bool now = d2 < hin2 && d2 < hjn * hjn;
        if (was == now) return;
        if (!reports(R, true, s, j, noi[j])) return;
        const int k = atomicAdd(ctr, 1);
        if (k < cap) ev[k] = make_int2(now ? (int)s : ~(int)s, j);
        else ctr[1] = 1;
    }
};

__global__ void __launch_bounds__(kBandBlock) k_band_events(TreeDev T, const double* __restrict__ sx,
                                                            const double* __restrict__ sy,
                                                            const double* __restrict__ sz,
                                                            const double* __restrict__ h,
                                                            const double* __restrict__ hnew,
                                                            const int* __restrict__ noi,
                                                            const int* __restrict__ nbr, int maxnb, BandRule R,
                                                            const int* __restrict__ list,
                                                            const int* __restrict__ list_count,
                                                            const float* __restrict__ node_hmax, int2* ev, int cap,
                                                            int* ctr, DevStatus* st) {
    __shared__ EventSmem smem[kBandWarps][4];
    if (st->code) return;
    const long cnt = *list_count;
    if (cnt == 0) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sg = lane >> 3, r = lane & 7;
    EventSmem* m = &smem[w][sg];
    const long nwarps = (long)gridDim.x * kBandWarps;
    for (long gw = ((long)blockIdx.x * kBandBlock + threadIdx.x) >> 5; gw * 4 < cnt; gw += nwarps) {
        const long q = gw * 4 + sg;
        const bool valid = q < cnt;
        const int s = valid ? list[q] : 0;
        const double px = sx[s], py = sy[s], pz = sz[s], hio = h[s], hin = hnew[s];
        const int ni = noi[s];
        const bool below = ni < R.target;
        if (valid && !below) {
            // above the band: the pairs it loses, from its list
            const double hin2 = hin * hin;
            for (int k = r; k < min(ni, maxnb); k += 8) {
                const int j = nbr[nb_index(s, k, maxnb)];
                const double d2 = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
                const double hjn = hnew[j];
                if (d2 < hin2 && d2 < hjn * hjn) continue;  // still a pair
                if (!reports(R, false, s, j, noi[j])) continue;
                const int e = atomicAdd(ctr, 1);
                if (e < cap) ev[e] = make_int2(~s, j);
                else ctr[1] = 1;
            }
        }
        EventVisit v{sx, sy, sz, h, hnew, noi, R, px, py, pz, hio * hio, hin * hin, (long)s, ev, cap, ctr};
        const bool walk = valid && below;
        band_walk(T, M, walk, px, py, pz, walk ? fmax(hio, hin) : -1.0, node_hmax, m->stk, m->rf, m->re, st, v);
        __syncwarp();
    }
}

__device__ __forceinline__ bool tombstone(int* nbr, const int* noi, int maxnb, int a, int b) {
    const int k = min(noi[a], maxnb);
    for (int q = 0; q < k; ++q) {
        const size_t ix = nb_index(a, q, maxnb);
        if (nbr[ix] == b) {
            nbr[ix] = -1;
            return true;
        }
    }
    return false;
}

__global__ void k_band_remove(const int2* __restrict__ ev, const int* __restrict__ ctr, int cap, int* nbr,
                              const int* __restrict__ noi, int maxnb, int* dirty, DevStatus* st) {
    if (ctr[1]) return;
    const int m = min(ctr[0], cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const int2 v = ev[e];
        if (v.x >= 0) continue;
        const int i = ~v.x, j = v.y;
        const bool a = tombstone(nbr, noi, maxnb, i, j);
        const bool b = tombstone(nbr, noi, maxnb, j, i);
        if (!a || !b) set_status(st, MHPC_ERR_NEIGHBOURS, i);  // lists and h disagree: cannot happen
        dirty[i] = 1;
        dirty[j] = 1;
    }
}

__global__ void k_band_compact(int n, const int* __restrict__ ctr, int* nbr, int* noi, int maxnb, int* dirty) {
    if (ctr[1]) return;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        if (!dirty[a]) continue;
        dirty[a] = 0;
        const int k = min(noi[a], maxnb);
        int w = 0;
        for (int q = 0; q < k; ++q) {
            const int v = nbr[nb_index(a, q, maxnb)];
            if (v >= 0) nbr[nb_index(a, w++, maxnb)] = v;
        }
        noi[a] = w;
    }
}

__device__ __forceinline__ void append(int* nbr, int* noi, int maxnb, int a, int b, DevStatus* st) {
    const int k = atomicAdd(noi + a, 1);
    if (k < maxnb) nbr[nb_index(a, k, maxnb)] = b;
    else set_status(st, MHPC_ERR_NEIGHBOURS, a);
}

__global__ void k_band_add(const int2* __restrict__ ev, const int* __restrict__ ctr, int cap, int* nbr, int* noi,
                           int maxnb, DevStatus* st) {
    if (ctr[1]) return;
    const int m = min(ctr[0], cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const int2 v = ev[e];
        if (v.x < 0) continue;
        append(nbr, noi, maxnb, v.x, v.y, st);
        append(nbr, noi, maxnb, v.y, v.x, st);
    }
}

// The round's new h, or (event buffer overflow: no list was edited) the old
// ones back into hnew.
__global__ void k_band_commit(const int* __restrict__ list, const int* __restrict__ list_count,
                              const int* __restrict__ ctr, double* h, double* hnew, DevStatus* st) {
    const int m = *list_count;
    const bool ok = ctr[1] == 0;
    if (!ok && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->sml_band_skipped, 1);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int i = list[q];
        if (ok) h[i] = hnew[i];
        else hnew[i] = h[i];
    }
}

__global__ void k_copy_h(int n, const double* __restrict__ a, double* b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

}  // namespace

int sph_band_fixup(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                   double* h, int* nbr, int* noi, const BandBuffers& B, int target, int tol, int rounds,
                   DevStatus* st, cudaStream_t s) {
    if (P.n <= 0 || rounds <= 0) return MHPC_OK;
    const int n = P.n;
    const int g = grid_for(n, 256, 148 * 16);
    const int* list_count = B.off + n;
    BandRule R{target, tol};
    CUDA_TRY(cudaMemsetAsync(B.dirty, 0, sizeof(int) * n, s));
    k_copy_h<<<g, 256, 0, s>>>(n, h, B.hnew);
    k_copy_h<<<g, 256, 0, s>>>(n, h, B.h0);
    for (int r = 0; r < rounds; ++r) {
        k_band_flags<<<g, 256, 0, s>>>(n, noi, R, B.flags);
        int rc = scan_exclusive_i32(B.flags, B.off, n, B.scan_scratch, s);
        if (rc) return rc;
        k_band_compact_list<<<g, 256, 0, s>>>(n, B.flags, B.off, B.list, B.ctr, st, r);
        k_band_select<<<148 * 8, kBandBlock, 0, s>>>(T, x, y, z, h, B.h0, noi, nbr, P.maxnb, B.list, list_count, R,
                                                     B.hnew, T.hmax, st);
        k_band_events<<<148 * 8, kBandBlock, 0, s>>>(T, x, y, z, h, B.hnew, noi, nbr, P.maxnb, R, B.list, list_count,
                                                     T.hmax, B.events, B.cap_events, B.ctr, st);
        k_band_remove<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, nbr, noi, P.maxnb, B.dirty, st);
        k_band_compact<<<g, 256, 0, s>>>(n, B.ctr, nbr, noi, P.maxnb, B.dirty);
        k_band_add<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, nbr, noi, P.maxnb, st);
        k_band_commit<<<148 * 4, 256, 0, s>>>(B.list, list_count, B.ctr, h, B.hnew, st);
    }
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
