// Stable LSD radix sort of (64-bit key, 32-bit value) pairs and a device-wide
// exclusive scan.
//
// The reference sorts with cub::DeviceRadixSort::SortPairs and a cudaMalloc /
// cudaFree of temporary storage on every call (src/helper.cu:150-166).  This
// sort is the library's own: one read of the keys builds all eight 8-bit digit
// histograms, then each pass is a single "onesweep" kernel (tile ranking with
// warp ballots, decoupled look-back across tiles, shared-memory staging so
// that the scatter writes runs of equal digits contiguously).  Scratch is
// caller-provided; nothing is allocated per call.  Sorting is stable, so equal
// keys keep ascending input position, which is the contract of the CUB call it
// replaces.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kRadixBits = 8;
constexpr int kRadix = 256;
constexpr int kPasses = 8;
constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kItems = 16;
constexpr int kTile = kBlock * kItems;  // 4096
constexpr unsigned long long kFlagAgg = 1ULL << 62;
constexpr unsigned long long kFlagInc = 2ULL << 62;
constexpr long kSpinLimit = 1L << 22;

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct SortScratch {
    uint64_t* keys_tmp;
    int* vals_tmp;
    unsigned* hist;                 // [kPasses][kRadix] counts, then exclusive bases
    unsigned* tile_counter;         // [kPasses]
    unsigned long long* look;       // [kPasses][ntiles][kRadix]
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static SortScratch carve(void* base, int n) {
    char* p = (char*)base;
    SortScratch s;
    s.keys_tmp = (uint64_t*)p; p += align256(sizeof(uint64_t) * (size_t)n);
    s.vals_tmp = (int*)p; p += align256(sizeof(int) * (size_t)n);
    s.hist = (unsigned*)p; p += align256(sizeof(unsigned) * kPasses * kRadix);
    s.tile_counter = (unsigned*)p; p += align256(sizeof(unsigned) * kPasses);
    s.look = (unsigned long long*)p;
    return s;
}

// Lanes of the warp holding the same 8-bit digit d: eight ballots, one per
// digit bit (on B200 cheaper than a match instruction unless most lanes share
// the digit).  Every lane of the warp must call it.
__device__ __forceinline__ unsigned digit_peers(unsigned d) {
    unsigned peers = MHPC_FULL;
#pragma unroll
    for (int b = 0; b < kRadixBits; ++b) {
        const unsigned bb = __ballot_sync(MHPC_FULL, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? bb : ~bb;
    }
    return peers;
}

// All eight digit histograms in one read of the keys: plain shared-memory
// atomics per key and digit (same-address conflicts within a warp are
// resolved by the hardware faster than aggregating them first), then one
// global atomic per bin per block.
__global__ void __launch_bounds__(kBlock) k_hist(const uint64_t* __restrict__ keys, int n, unsigned* hist) {
    __shared__ unsigned sh[kPasses * kRadix];
    for (int i = threadIdx.x; i < kPasses * kRadix; i += kBlock) sh[i] = 0;
    __syncthreads();
    long stride = (long)gridDim.x * kBlock;
    for (long i = (long)blockIdx.x * kBlock + threadIdx.x; i < n; i += stride) {
        const uint64_t k = __ldg(keys + i);
#pragma unroll
        for (int p = 0; p < kPasses; ++p)
            atomicAdd(&sh[p * kRadix + ((unsigned)(k >> (p * kRadixBits)) & (kRadix - 1))], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPasses * kRadix; i += kBlock)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of each pass's 256-bin histogram, in place.
__global__ void __launch_bounds__(kRadix) k_hist_scan(unsigned* hist) {
    __shared__ unsigned s[kRadix];
    unsigned* h = hist + blockIdx.x * kRadix;
    unsigned v = h[threadIdx.x];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
        unsigned t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    h[threadIdx.x] = s[threadIdx.x] - v;
}

struct OnesweepSmem {
    unsigned whist[kWarps][kRadix];
    unsigned tile_off[kRadix];
    unsigned gbase[kRadix];
    unsigned tile_id;
    uint64_t keys[kTile];
    int vals[kTile];
};

__global__ void __launch_bounds__(kBlock, 2)
k_onesweep(const uint64_t* __restrict__ kin, const int* __restrict__ vin, uint64_t* __restrict__ kout,
           int* __restrict__ vout, int n, int pass, const unsigned* __restrict__ digit_base,
           unsigned* tile_counter, unsigned long long* look, DevStatus* st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    OnesweepSmem& S = *reinterpret_cast<OnesweepSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int shift = pass * kRadixBits;
    if (tid == 0) S.tile_id = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < kWarps * kRadix; i += kBlock) (&S.whist[0][0])[i] = 0;
    __syncthreads();
    const long tile = S.tile_id;
    const long ntiles = ((long)n + kTile - 1) / kTile;
    const long base = tile * kTile + (long)warp * (32 * kItems);

    uint64_t key[kItems];
    int val[kItems];
    unsigned rank[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        long idx = base + i * 32 + lane;
        if (idx < n) {
            key[i] = __ldg(kin + idx);
            val[i] = vin ? __ldg(vin + idx) : (int)idx;
        } else {
            key[i] = 0;
            val[i] = 0;
        }
    }
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        long idx = base + i * 32 + lane;
        bool valid = idx < n;
        unsigned vm = __ballot_sync(MHPC_FULL, valid);
        unsigned d = (unsigned)(key[i] >> shift) & (kRadix - 1);
        unsigned peers = digit_peers(d) & vm;
        if (!valid) peers = 1u << lane;
        int leader = __ffs(peers) - 1;
        unsigned b = 0;
        if (valid && lane == leader) b = S.whist[warp][d];
        b = __shfl_sync(MHPC_FULL, b, leader);
        rank[i] = b + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == leader) S.whist[warp][d] = b + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: prefix over warps, tile total, look-back, global base
    {
        const int d = tid;
        unsigned run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            unsigned c = S.whist[w][d];
            S.whist[w][d] = run;
            run += c;
        }
        unsigned long long* mine = look + ((long)pass * ntiles + tile) * kRadix + d;
        unsigned long long excl = 0;
        if (tile == 0) {
            st_relaxed(mine, kFlagInc | (unsigned long long)run);
        } else {
            st_relaxed(mine, kFlagAgg | (unsigned long long)run);
            long j = tile - 1;
            long spins = 0;
            while (j >= 0) {
                unsigned long long v = ld_relaxed(look + ((long)pass * ntiles + j) * kRadix + d);
                unsigned long long f = v & (3ULL << 62);
                if (f == 0) {
                    if (++spins > kSpinLimit) {
                        set_status(st, MHPC_ERR_TIMEOUT, 100 + pass);
                        break;
                    }
                    continue;
                }
                excl += v & 0xffffffffULL;
                if (f == kFlagInc) break;
                --j;
            }
            st_relaxed(mine, kFlagInc | (excl + run));
        }
        S.gbase[d] = digit_base[pass * kRadix + d] + (unsigned)excl;
        // exclusive scan of tile totals over digits (block-wide, 256 = kBlock)
        S.tile_off[d] = run;
    }
    __syncthreads();
    {
        // Hillis-Steele in place over 256 entries
        unsigned v = S.tile_off[tid];
        unsigned incl = v;
        for (int o = 1; o < kRadix; o <<= 1) {
            unsigned t = tid >= o ? S.tile_off[tid - o] : 0;
            __syncthreads();
            incl += t;
            S.tile_off[tid] = incl;
            __syncthreads();
        }
        S.tile_off[tid] = incl - v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        long idx = base + i * 32 + lane;
        if (idx < n) {
            unsigned d = (unsigned)(key[i] >> shift) & (kRadix - 1);
            unsigned pos = S.tile_off[d] + S.whist[warp][d] + rank[i];
            S.keys[pos] = key[i];
            S.vals[pos] = val[i];
        }
    }
    __syncthreads();
    long tile_count = (long)n - tile * kTile;
    if (tile_count > kTile) tile_count = kTile;
    for (int q = tid; q < tile_count; q += kBlock) {
        uint64_t k = S.keys[q];
        unsigned d = (unsigned)(k >> shift) & (kRadix - 1);
        unsigned dest = S.gbase[d] + (q - S.tile_off[d]);
        kout[dest] = k;
        vout[dest] = S.vals[q];
    }
}

// ------------------------------------------------------------------ scan
constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanBlock * kScanItems;

__device__ __forceinline__ int block_excl_scan(int v, int* sw, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(MHPC_FULL, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) sw[w] = x;
    __syncthreads();
    if (w == 0) {
        int y = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(MHPC_FULL, y, o);
            if (lane >= o) y += t;
        }
        sw[lane] = y;
    }
    __syncthreads();
    int before = w > 0 ? sw[w - 1] : 0;
    *total = sw[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_reduce(const int* __restrict__ in, int n, int* bsum) {
    __shared__ int sw[32];
    long base = (long)blockIdx.x * kScanChunk;
    int s = 0;
    for (int i = 0; i < kScanItems; ++i) {
        long idx = base + i * kScanBlock + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    int tot;
    block_excl_scan(s, sw, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_bsum(int* bsum, int nb) {
    __shared__ int sw[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += 1024) {
        int i = b0 + threadIdx.x;
        int v = i < nb ? bsum[i] : 0;
        int tot;
        int e = block_excl_scan(v, sw, &tot);
        if (i < nb) bsum[i] = carry + e;
        carry += tot;
    }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_down(const int* __restrict__ in, int* out, int n,
                                                          const int* __restrict__ bsum) {
    __shared__ int sw[32];
    __shared__ int tile[kScanChunk];
    long base = (long)blockIdx.x * kScanChunk;
    for (int i = 0; i < kScanItems; ++i) {
        long idx = base + i * kScanBlock + threadIdx.x;
        tile[i * kScanBlock + threadIdx.x] = idx < n ? in[idx] : 0;
    }
    __syncthreads();
    int loc[kScanItems];
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        loc[i] = s;
        s += tile[threadIdx.x * kScanItems + i];
    }
    int tot;
    int e = block_excl_scan(s, sw, &tot);
    int carry = bsum[blockIdx.x] + e;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) tile[threadIdx.x * kScanItems + i] = carry + loc[i];
    __syncthreads();
    for (int i = 0; i < kScanItems; ++i) {
        long idx = base + i * kScanBlock + threadIdx.x;
        if (idx < n) out[idx] = tile[i * kScanBlock + threadIdx.x];
    }
}

__global__ void k_scan_total(const int* __restrict__ in, int* out, int n) {
    // out[n] = out[n-1] + in[n-1]
    if (n > 0) out[n] = out[n - 1] + in[n - 1];
    else out[0] = 0;
}

constexpr size_t align256c(size_t b) { return (b + 255) & ~size_t(255); }

constexpr size_t scratch_formula(long n) {
    return align256c(sizeof(uint64_t) * (size_t)n) + align256c(sizeof(int) * (size_t)n) +
           align256c(sizeof(unsigned) * kPasses * kRadix) + align256c(sizeof(unsigned) * kPasses) +
           align256c(sizeof(unsigned long long) * kPasses * (size_t)(((n + kTile - 1) / kTile) < 1 ? 1 : ((n + kTile - 1) / kTile)) * kRadix);
}

}  // namespace

size_t sort_scratch_bytes(int n) { return scratch_formula(n); }

int sort_pairs_u64(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out, int* vals_out, int n,
                   void* scratch, size_t scratch_bytes, DevStatus* st, cudaStream_t s) {
    if (n < 0) return MHPC_ERR_ARG;
    if (n == 0) return MHPC_OK;
    if (!keys_in || !keys_out || !vals_out) return MHPC_ERR_ARG;
    if (!scratch || scratch_bytes < sort_scratch_bytes(n)) return MHPC_ERR_ARG;
    SortScratch S = carve(scratch, n);
    long ntiles = ((long)n + kTile - 1) / kTile;
    // zero histograms, tile counters and look-back words in one memset
    size_t zero_bytes = sort_scratch_bytes(n) - ((char*)S.hist - (char*)scratch);
    CUDA_TRY(cudaMemsetAsync(S.hist, 0, zero_bytes, s));
    k_hist<<<grid_for(n, kBlock, 148 * 4), kBlock, 0, s>>>(keys_in, n, S.hist);
    CUDA_TRY(cudaGetLastError());
    k_hist_scan<<<kPasses, kRadix, 0, s>>>(S.hist);
    CUDA_TRY(cudaGetLastError());
    // per device (a process may drive several GPUs); a cheap host call
    size_t smem = sizeof(OnesweepSmem);
    CUDA_TRY(cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t* kin = keys_in;
    const int* vin = vals_in;
    for (int p = 0; p < kPasses; ++p) {
        uint64_t* kout = (p & 1) ? keys_out : S.keys_tmp;
        int* vout = (p & 1) ? vals_out : S.vals_tmp;
        k_onesweep<<<(int)ntiles, kBlock, smem, s>>>(kin, vin, kout, vout, n, p, S.hist, S.tile_counter + p,
                                                      S.look, st);
        CUDA_TRY(cudaGetLastError());
        kin = kout;
        vin = vout;
    }
    return MHPC_OK;
}

// ------------------------------------------------- sort without allocation
// Some callers cannot allocate device memory: applications whose own pool
// reserves the device's memory at start-up (a cudaMalloc would fail or
// fragment it) and services that forbid allocation after initialisation.
// For them mhpc_sort_pairs_noalloc keeps its scratch in this file-scope
// device array, sized for kNoAllocMaxN keys.  Every GPU that loads the
// library holds the array until the process exits.
constexpr long kNoAllocMaxN = 1L << 20;
constexpr size_t kNoAllocStatusBytes = 256;
constexpr size_t kNoAllocBytes = scratch_formula(kNoAllocMaxN) + kNoAllocStatusBytes;
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocBytes];

namespace {

__global__ void k_copy_status(const DevStatus* st, int* out) { *out = st->code; }

// Device address of g_noalloc_sort_scratch on the current device.  The host
// symbol is only a stand-in for the device array, so the address is looked up
// once per device with that device current and cached.
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[256];

int noalloc_scratch(void** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return MHPC_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_sort_scratch) != cudaSuccess || !p) return MHPC_ERR_CUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return MHPC_OK;
}

}  // namespace

extern "C" int mhpc_sort_noalloc_max_n(void) { return (int)kNoAllocMaxN; }

extern "C" int mhpc_sort_pairs_noalloc(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out,
                                       int* vals_out, int n, int* status_dev, void* stream) {
    if (n < 0) return MHPC_ERR_ARG;
    if (n > kNoAllocMaxN) return MHPC_ERR_CAPACITY;
    cudaStream_t s = (cudaStream_t)stream;
    void* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    DevStatus* st = reinterpret_cast<DevStatus*>((char*)base + kNoAllocBytes - kNoAllocStatusBytes);
    CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(DevStatus), s));
    if (n > 0) {
        // sort_pairs_u64 clears the histograms, tile counters and look-back
        // words it needs before its first kernel
        rc = sort_pairs_u64(keys_in, vals_in, keys_out, vals_out, n, base, kNoAllocBytes - kNoAllocStatusBytes,
                            st, s);
        if (rc) return rc;
    }
    if (status_dev) {
        k_copy_status<<<1, 1, 0, s>>>(st, status_dev);
        CUDA_TRY(cudaGetLastError());
    }
    return MHPC_OK;
}

size_t scan_scratch_bytes(int n) {
    long nb = ((long)n + kScanChunk - 1) / kScanChunk;
    if (nb < 1) nb = 1;
    return align256(sizeof(int) * (size_t)nb);
}

int scan_exclusive_i32(const int* in, int* out, int n, void* scratch, cudaStream_t s) {
    if (n <= 0) {
        CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int), s));
        return MHPC_OK;
    }
    int nb = (int)(((long)n + kScanChunk - 1) / kScanChunk);
    int* bsum = (int*)scratch;
    k_scan_reduce<<<nb, kScanBlock, 0, s>>>(in, n, bsum);
    k_scan_bsum<<<1, 1024, 0, s>>>(bsum, nb);
    k_scan_down<<<nb, kScanBlock, 0, s>>>(in, out, n, bsum);
    k_scan_total<<<1, 1, 0, s>>>(in, out, n);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
