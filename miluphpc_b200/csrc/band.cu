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
// k_band_select (selection, one warp per particle: a tree walk below the band,
// the particle's own list above it), k_band_events (one event per changed
// pair, likewise), k_band_mark + k_band_filter (removals: the marked lists
// re-tested with the new h), k_band_add, k_band_commit.  Every kernel after the
// compaction reads the list length on the device and returns at once when it
// is zero, so the host enqueues all rounds without synchronising.
#include "sph.cuh"
#include "walk.cuh"

namespace {

constexpr int kBandBlock = 128;  // 4 warps, one particle per warp
constexpr int kBandWarps = kBandBlock / 32;
constexpr int kBandCap = 256;    // candidates held per particle during the selection
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
    int stk[kWalkStack];
    int rf[32], re[32];
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
// reads them from the list instead of walking the tree.  A particle below the
// band whose search radius is capped at its current h (h already twice the
// h of the first round) cannot gain a pair: it keeps h without a walk.  A
// new h above the old one raises the largest-h bounds of the particle's leaf
// and ancestors (grow-only).
__global__ void __launch_bounds__(kBandBlock) k_band_select(TreeDev T, const double* __restrict__ sx,
                                                            const double* __restrict__ sy,
                                                            const double* __restrict__ sz,
                                                            const double* __restrict__ h,
                                                            const double* __restrict__ h0,
                                                            const int* __restrict__ noi,
                                                            const int* __restrict__ nbr, int maxnb,
                                                            const int* __restrict__ list,
                                                            const int* __restrict__ list_count, BandRule R,
                                                            const long long* __restrict__ ord, double* hnew,
                                                            float* node_hmax, DevStatus* st) {
    __shared__ SelectSmem smem[kBandWarps];
    if (st->code) return;
    const long cnt = *list_count;
    if (cnt == 0) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    SelectSmem* m = &smem[w];
    const long nwarps = (long)gridDim.x * kBandWarps;
    for (long q = ((long)blockIdx.x * kBandBlock + threadIdx.x) >> 5; q < cnt; q += nwarps) {
        const int s = list[q];
        const double px = sx[s], py = sy[s], pz = sz[s], hi = h[s];
        const int ni = noi[s];
        const int want = R.want(ni);
        const bool above = ni >= R.target + R.tol;
        // from below at most twice the h before the first round (at a free
        // surface the neighbours' h may not reach the particle at all), and
        // never past the edge of the bounding box
        const double hcap = ord_to_dbl(ord[1]) - ord_to_dbl(ord[0]);
        double rad = above ? R.radius(ni, hi) : fmin(fmin(R.radius(ni, hi), 2.0 * h0[s]), hcap);
        // the list holds the candidates of a particle above the band
        const bool from_list = above && ni <= min(maxnb, kBandCap);
        bool done = !above && rad <= hi;  // capped: nothing to gain
        double result = hi;
        for (int attempt = 0; attempt < 5 && !done; ++attempt) {
            if (lane == 0) m->cnt = from_list ? ni : 0;
            __syncwarp();
            if (from_list) {
                for (int k = lane; k < ni; k += 32) {
                    const int j = nbr[nb_index(s, k, maxnb)];
                    m->d2[k] = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
                }
            } else {
                SelectVisit v{sx, sy, sz, h, px, py, pz, rad * rad, (long)s, m};
                warp_walk(T, M, true, px, py, pz, rad, node_hmax, m->stk, m->rf, m->re, st, v);
            }
            __syncwarp();
            const int found = m->cnt;
            if (found > kBandCap) {
                rad = 0.8 * rad;
                continue;
            }
            if (found > want) {
                // ranks by counting (d2 ascending; equal distances have equal values,
                // so the two order statistics do not depend on how ties are broken)
                double lo = -1.0, hi2 = -1.0;
                for (int a = lane; a < found; a += 32) {
                    const double da = m->d2[a];
                    int rank = 0;
                    for (int b = 0; b < found; ++b) {
                        const double db = m->d2[b];
                        rank += (db < da) || (db == da && b < a);
                    }
                    if (rank == want - 1) lo = da;
                    if (rank == want) hi2 = da;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    lo = fmax(lo, __shfl_xor_sync(MHPC_FULL, lo, o));
                    hi2 = fmax(hi2, __shfl_xor_sync(MHPC_FULL, hi2, o));
                }
                result = 0.5 * (sqrt(lo) + sqrt(hi2));
            } else {
                result = rad;
            }
            done = true;
        }
        // still more than kBandCap candidates after the last shrink: unchanged
        if (lane == 0) {
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
    int stk[kWalkStack];
    int rf[32], re[32];
};

// Who reports a pair whose status changes.  Only particles whose h changed
// in this round report: one above the band lowers its h, so it only loses
// pairs, all of them in its list; one below raises it and walks the tree for
// the pairs it gains or loses.  A pair with one changed end is reported by
// that end; of two changed ends of the same kind, by the smaller index; of a
// lowered and a raised end, by the raised one (its walk sees every pair the
// other's list can miss).
__device__ __forceinline__ bool reports(bool i_raised, long i, int j, const double* h, const double* hn) {
    const double hj = h[j], hjn = hn[j];
    if (hjn == hj) return true;
    const bool j_raised = hjn > hj;
    if (i_raised != j_raised) return i_raised;
    return i < j;
}

// Pair changes of a particle whose h rose: every j within h_i' (> h_i) with
// d < max(h_j, h_j'); the pair is present before when d < min(h_i, h_j) and
// after when d < min(h_i', h_j') (the list walk's test, d^2 against h^2).
struct EventVisit {
    const double *sx, *sy, *sz, *h, *hn;
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
        if (!reports(true, s, j, h, hn)) return;
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
                                                            const int* __restrict__ nbr, int maxnb,
                                                            const int* __restrict__ list,
                                                            const int* __restrict__ list_count,
                                                            const float* __restrict__ node_hmax, int2* ev, int cap,
                                                            int* ctr, DevStatus* st, const int* skip = nullptr) {
    __shared__ EventSmem smem[kBandWarps];
    if (st->code) return;
    if (skip && *skip) return;  // lists truncated: the caller re-walks them instead
    const long cnt = *list_count;
    if (cnt == 0) return;
    const int M = *T.nodes;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    EventSmem* m = &smem[w];
    const long nwarps = (long)gridDim.x * kBandWarps;
    for (long q = ((long)blockIdx.x * kBandBlock + threadIdx.x) >> 5; q < cnt; q += nwarps) {
        const int s = list[q];
        const double px = sx[s], py = sy[s], pz = sz[s], hio = h[s], hin = hnew[s];
        if (hin == hio) continue;  // unchanged: its partners report
        if (hin < hio) {
            // lowered: the pairs it loses, from its list
            const int ni = min(noi[s], maxnb);
            const double hin2 = hin * hin;
            for (int k = lane; k < ni; k += 32) {
                const int j = nbr[nb_index(s, k, maxnb)];
                const double d2 = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
                const double hjn = hnew[j];
                if (d2 < hin2 && d2 < hjn * hjn) continue;  // still a pair
                if (!reports(false, s, j, h, hnew)) continue;
                const int e = atomicAdd(ctr, 1);
                if (e < cap) ev[e] = make_int2(~s, j);
                else ctr[1] = 1;
            }
        } else {
            EventVisit v{sx, sy, sz, h, hnew, px, py, pz, hio * hio, hin * hin, (long)s, ev, cap, ctr};
            warp_walk(T, M, true, px, py, pz, hin, node_hmax, m->stk, m->rf, m->re, st, v);
        }
        __syncwarp();
    }
}

// Removals: both ends of every removal event are marked; each marked list is
// then filtered with the pair test of the new h (d < min(h_i', h_j'), the list
// walk's test), which drops exactly the pairs the events removed (every pair
// in a list was present with the old h, and a pair whose status did not change
// passes).  One warp per marked list, order kept (ballot compaction).
__global__ void k_band_mark(const int2* __restrict__ ev, const int* __restrict__ ctr, int cap, int* dirty,
                            const int* skip = nullptr) {
    if (ctr[1] || (skip && *skip)) return;
    const int m = min(ctr[0], cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const int2 v = ev[e];
        if (v.x >= 0) continue;
        dirty[~v.x] = 1;
        dirty[v.y] = 1;
    }
}

__global__ void k_band_filter(int n, const int* __restrict__ ctr, const double* __restrict__ sx,
                              const double* __restrict__ sy, const double* __restrict__ sz,
                              const double* __restrict__ hn, int* nbr, int* noi, int maxnb, int* dirty,
                              const int* skip = nullptr) {
    if (ctr[1] || (skip && *skip)) return;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = warp * 32; base < n; base += nwarps * 32) {
        const long me = base + lane;
        const bool mark = me < n && dirty[me];
        unsigned todo = __ballot_sync(MHPC_FULL, mark);
        if (mark) dirty[me] = 0;
        while (todo) {
            const int b = __ffs(todo) - 1;
            todo &= todo - 1;
            const long a = base + b;
            const int k = min(noi[a], maxnb);
            const double px = sx[a], py = sy[a], pz = sz[a], ha = hn[a];
            const double ha2 = ha * ha;
            int w = 0;
            for (int q0 = 0; q0 < k; q0 += 32) {
                const int q = q0 + lane;
                int j = -1;
                bool keep = false;
                if (q < k) {
                    j = nbr[nb_index(a, q, maxnb)];
                    const double d2 = d2_exact(px - __ldg(sx + j), py - __ldg(sy + j), pz - __ldg(sz + j));
                    const double hj = hn[j];
                    keep = d2 < ha2 && d2 < hj * hj;
                }
                const unsigned bk = __ballot_sync(MHPC_FULL, keep);
                // entries are only moved towards the front: slot w + rank <= q
                __syncwarp();
                if (keep) nbr[nb_index(a, w + __popc(bk & lt), maxnb)] = j;
                w += __popc(bk);
                __syncwarp();
            }
            if (lane == 0) noi[a] = w;
            __syncwarp();
        }
    }
}

// A list already holding maxnb entries: an error for the band repair (its
// targets stay far below maxnb); the variable-h iteration (trunc given) marks
// the lists truncated and re-walks them instead.
__device__ __forceinline__ void append(int* nbr, int* noi, int maxnb, int a, int b, DevStatus* st, int* trunc) {
    const int k = atomicAdd(noi + a, 1);
    if (k < maxnb) nbr[nb_index(a, k, maxnb)] = b;
    else if (trunc) *trunc = 1;
    else set_status(st, MHPC_ERR_NEIGHBOURS, a);
}

// Appends land in atomic order: both ends are marked in `appended` and their
// lists sorted afterwards (k_sort_appended), so that the lists, and the sums
// over them, do not depend on the order in which the events ran.
__global__ void k_band_add(const int2* __restrict__ ev, const int* __restrict__ ctr, int cap, int* nbr, int* noi,
                           int maxnb, DevStatus* st, int* appended, int* trunc = nullptr) {
    if (ctr[1] || (trunc && *trunc)) return;
    const int m = min(ctr[0], cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const int2 v = ev[e];
        if (v.x < 0) continue;
        append(nbr, noi, maxnb, v.x, v.y, st, trunc);
        append(nbr, noi, maxnb, v.y, v.x, st, trunc);
        appended[v.x] = 1;
        appended[v.y] = 1;
    }
}

// Every list marked in `appended` sorted by neighbour index (one warp per
// list: ranks by counting, the entries are distinct), and the mark cleared.
constexpr int kSortPerLane = 8;  // lists up to 256 entries in registers; longer ones by lane 0
__global__ void k_sort_appended(int n, int* appended, int* nbr, const int* __restrict__ noi, int maxnb) {
    const int lane = threadIdx.x & 31;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = warp * 32; base < n; base += nwarps * 32) {
        const long me = base + lane;
        const bool mark = me < n && appended[me];
        unsigned todo = __ballot_sync(MHPC_FULL, mark);
        if (mark) appended[me] = 0;
        while (todo) {
            const int b = __ffs(todo) - 1;
            todo &= todo - 1;
            const long a = base + b;
            const int k = min(noi[a], maxnb);
            if (k <= 32 * kSortPerLane) {
                int val[kSortPerLane], rank[kSortPerLane];
#pragma unroll
                for (int r = 0; r < kSortPerLane; ++r) {
                    const int q = lane + 32 * r;
                    val[r] = q < k ? nbr[nb_index(a, q, maxnb)] : 0;
                    rank[r] = 0;
                }
                for (int q = 0; q < k; ++q) {
                    const int v = nbr[nb_index(a, q, maxnb)];
#pragma unroll
                    for (int r = 0; r < kSortPerLane; ++r) rank[r] += v < val[r];
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < kSortPerLane; ++r)
                    if (lane + 32 * r < k) nbr[nb_index(a, rank[r], maxnb)] = val[r];
            } else if (lane == 0) {
                for (int q = 1; q < k; ++q) {  // insertion sort in place
                    const int v = nbr[nb_index(a, q, maxnb)];
                    int w = q;
                    while (w > 0 && nbr[nb_index(a, w - 1, maxnb)] > v) {
                        nbr[nb_index(a, w, maxnb)] = nbr[nb_index(a, w - 1, maxnb)];
                        --w;
                    }
                    nbr[nb_index(a, w, maxnb)] = v;
                }
            }
            __syncwarp();
        }
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

__global__ void k_reset_events(int* ctr) {
    ctr[0] = 0;
    ctr[1] = 0;
}

}  // namespace

int sph_sort_appended(const SphParams& P, int* nbr, const int* noi, int* appended, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    k_sort_appended<<<148 * 4, 256, 0, s>>>(P.n, appended, nbr, noi, P.maxnb);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int sph_apply_h_changes(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                        const double* h, const double* hnew, int* nbr, int* noi, const int* list,
                        const int* list_count, const BandBuffers& B, int* trunc, DevStatus* st, cudaStream_t s) {
    if (P.n <= 0) return MHPC_OK;
    const int g = grid_for(P.n, 256, 148 * 16);
    k_reset_events<<<1, 1, 0, s>>>(B.ctr);
    k_band_events<<<148 * 8, kBandBlock, 0, s>>>(T, x, y, z, h, hnew, noi, nbr, P.maxnb, list, list_count, T.hmax,
                                                 B.events, B.cap_events, B.ctr, st, trunc);
    k_band_mark<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, B.dirty, trunc);
    k_band_filter<<<148 * 8, 128, 0, s>>>(P.n, B.ctr, x, y, z, hnew, nbr, noi, P.maxnb, B.dirty, trunc);
    k_band_add<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, nbr, noi, P.maxnb, st, B.appended, trunc);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

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
                                                     P.ord, B.hnew, T.hmax, st);
        k_band_events<<<148 * 8, kBandBlock, 0, s>>>(T, x, y, z, h, B.hnew, noi, nbr, P.maxnb, B.list, list_count,
                                                     T.hmax, B.events, B.cap_events, B.ctr, st);
        k_band_mark<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, B.dirty);
        k_band_filter<<<148 * 8, 128, 0, s>>>(n, B.ctr, x, y, z, B.hnew, nbr, noi, P.maxnb, B.dirty);
        k_band_add<<<148 * 4, 256, 0, s>>>(B.events, B.ctr, B.cap_events, nbr, noi, P.maxnb, st, B.appended);
        k_band_commit<<<148 * 4, 256, 0, s>>>(B.list, list_count, B.ctr, h, B.hnew, st);
    }
    k_sort_appended<<<148 * 4, 256, 0, s>>>(n, B.appended, nbr, noi, P.maxnb);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
