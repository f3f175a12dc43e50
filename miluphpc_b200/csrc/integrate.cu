// FP64 state update, gather/scatter between the caller's particle order and
// the SFC-sorted working order, diagnostics, and FP64 direct summation.
#include "common.cuh"
#include "integrate.cuh"

namespace {

__global__ void __launch_bounds__(256) k_gather(int n, const int* __restrict__ perm, GatherList L) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = __ldg(perm + s);
#pragma unroll 4
        for (int a = 0; a < L.count; ++a) L.dst[a][s] = __ldg(L.src[a] + o);
        if (L.isrc) L.idst[s] = __ldg(L.isrc + o);
    }
}

__global__ void __launch_bounds__(256) k_scatter(int n, const int* __restrict__ perm, GatherList L) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = __ldg(perm + s);
#pragma unroll 4
        for (int a = 0; a < L.count; ++a) L.dst[a][o] = L.src[a][s];
    }
}

// LeapfrogNS::Kernel::updateX (src/integrator/device_leapfrog.cu:4-30)
__global__ void __launch_bounds__(256) k_leapfrog_x(mhpc_particles p, double dt) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        const double gx = p.g_ax[i], gy = p.g_ay[i], gz = p.g_az[i];
        p.x[i] += dt * (p.vx[i] + 0.5 * dt * gx);
        p.y[i] += dt * (p.vy[i] + 0.5 * dt * gy);
        p.z[i] += dt * (p.vz[i] + 0.5 * dt * gz);
        p.g_ax_old[i] = gx; p.g_ay_old[i] = gy; p.g_az_old[i] = gz;
    }
}

// LeapfrogNS::Kernel::updateV (device_leapfrog.cu:32-58)
__global__ void __launch_bounds__(256) k_leapfrog_v(mhpc_particles p, double dt) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        p.vx[i] += 0.5 * dt * (p.g_ax[i] + p.g_ax_old[i]);
        p.vy[i] += 0.5 * dt * (p.g_ay[i] + p.g_ay_old[i]);
        p.vz[i] += 0.5 * dt * (p.g_az[i] + p.g_az_old[i]);
    }
}

// ExplicitEulerNS::Kernel::update (src/integrator/device_explicit_euler.cu:4-54)
__global__ void __launch_bounds__(256) k_euler(mhpc_particles p, double dt, int gravity, int sph, int int_rho,
                                               int int_e, int int_sml) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        double ax = 0, ay = 0, az = 0;
        if (sph) { ax += p.ax[i]; ay += p.ay[i]; az += p.az[i]; }
        if (gravity) { ax += p.g_ax[i]; ay += p.g_ay[i]; az += p.g_az[i]; }
        p.vx[i] += dt * ax;
        p.vy[i] += dt * ay;
        p.vz[i] += dt * az;
        p.x[i] += dt * p.vx[i];
        p.y[i] += dt * p.vy[i];
        p.z[i] += dt * p.vz[i];
        if (int_rho) p.rho[i] = p.rho[i] + dt * p.drhodt[i];
        if (int_e) {
            p.e[i] += dt * p.dedt[i];
            if (p.e[i] < 1e-50) p.e[i] = 1e-50;
        }
        if (int_sml) p.sml[i] = p.sml[i] + dt * p.dsmldt[i];
    }
}

constexpr int kDiag = 11;

__global__ void __launch_bounds__(256) k_diag(mhpc_particles p, int sph, double* part) {
    double acc[kDiag];
#pragma unroll
    for (int k = 0; k < kDiag; ++k) acc[k] = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        const double m = p.mass[i], x = p.x[i], y = p.y[i], z = p.z[i];
        const double vx = p.vx[i], vy = p.vy[i], vz = p.vz[i];
        acc[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        if (sph && p.e) acc[1] += m * p.e[i];
        acc[2] += m * vx; acc[3] += m * vy; acc[4] += m * vz;
        acc[5] += m * (y * vz - z * vy);
        acc[6] += m * (z * vx - x * vz);
        acc[7] += m * (x * vy - y * vx);
        acc[8] += m * x; acc[9] += m * y; acc[10] += m * z;
    }
    __shared__ double sh[8][kDiag];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kDiag; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(MHPC_FULL, v, o);
        if (lane == 0) sh[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDiag) {
        double v = 0;
        for (int q = 0; q < 8; ++q) v += sh[q][threadIdx.x];
        part[blockIdx.x * kDiag + threadIdx.x] = v;
    }
}

__global__ void k_diag_final(int blocks, const double* part, double* out, const double* mass_total_part) {
    if (threadIdx.x < kDiag) {
        double v = 0;
        for (int b = 0; b < blocks; ++b) v += part[b * kDiag + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

// Direct summation: blockIdx.x covers 256 targets (one per thread), blockIdx.y
// a slice of the sources, staged 256 at a time in shared memory.
__global__ void __launch_bounds__(256) k_direct(const double* __restrict__ x, const double* __restrict__ y,
                                                const double* __restrict__ z, const double* __restrict__ m, int n,
                                                const int* __restrict__ tg, int nt, double eps2, double* gax,
                                                double* gay, double* gaz) {
    __shared__ double4 src[256];
    const int t = blockIdx.x * 256 + threadIdx.x;
    const bool valid = t < nt;
    const int ti = valid ? tg[t] : 0;
    const double px = x[ti], py = y[ti], pz = z[ti];
    const long per = ((long)n + gridDim.y - 1) / gridDim.y;
    const long j0 = (long)blockIdx.y * per;
    const long j1 = min((long)n, j0 + per);
    double ax = 0, ay = 0, az = 0;
    for (long b = j0; b < j1; b += 256) {
        const long j = b + threadIdx.x;
        __syncthreads();
        src[threadIdx.x] = j < j1 ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int cnt = (int)min((long)256, j1 - b);
        for (int q = 0; q < cnt; ++q) {
            const double4 s = src[q];
            const double dx = s.x - px, dy = s.y - py, dz = s.z - pz;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            if (b + q == ti || r2 <= 0.0) continue;
            const double ri = rsqrt(r2);
            const double f = s.w * ri * ri * ri;
            ax += f * dx; ay += f * dy; az += f * dz;
        }
    }
    if (valid) {
        atomicAdd(gax + t, ax);
        atomicAdd(gay + t, ay);
        atomicAdd(gaz + t, az);
    }
}

// FP32 FMA throughput probe: 8 independent dependent chains per thread.
constexpr int kFmaIters = 2048;
__global__ void __launch_bounds__(256) k_fma_peak(float* out, float b, float c) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < kFmaIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1234.5f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" int mhpc_fp32_peak(double* tflops) {
    if (!tflops) return MHPC_ERR_ARG;
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* out = nullptr;
    CUDA_TRY(cudaMalloc(&out, sizeof(float) * 65536));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 32;
    k_fma_peak<<<blocks, 256>>>(out, 0.999f, 1e-4f);  // warm up
    cudaEventRecord(e0);
    const int reps = 10;
    for (int r = 0; r < reps; ++r) k_fma_peak<<<blocks, 256>>>(out, 0.999f, 1e-4f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8 * kFmaIters * 256.0 * blocks * reps;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cudaGetLastError() == cudaSuccess ? MHPC_OK : MHPC_ERR_CUDA;
}

int launch_gather(int n, const int* perm, const GatherList& L, cudaStream_t s) {
    if (n <= 0 || (L.count == 0 && !L.isrc)) return MHPC_OK;
    k_gather<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, L);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_scatter(int n, const int* perm, const GatherList& L, cudaStream_t s) {
    if (n <= 0 || L.count == 0) return MHPC_OK;
    k_scatter<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, L);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_leapfrog_x(const mhpc_particles& p, double dt, cudaStream_t s) {
    k_leapfrog_x<<<grid_for(p.n, 256, 148 * 16), 256, 0, s>>>(p, dt);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_leapfrog_v(const mhpc_particles& p, double dt, cudaStream_t s) {
    k_leapfrog_v<<<grid_for(p.n, 256, 148 * 16), 256, 0, s>>>(p, dt);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_euler(const mhpc_particles& p, double dt, int gravity, int sph, int int_rho, int int_e, int int_sml,
                 cudaStream_t s) {
    k_euler<<<grid_for(p.n, 256, 148 * 16), 256, 0, s>>>(p, dt, gravity, sph, int_rho, int_e, int_sml);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_diagnostics(const mhpc_particles& p, int sph, double* part, double* out, cudaStream_t s) {
    const int blocks = 148 * 4;
    k_diag<<<blocks, 256, 0, s>>>(p, sph, part);
    k_diag_final<<<1, 32, 0, s>>>(blocks, part, out, nullptr);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

size_t diagnostics_scratch_doubles() { return 148 * 4 * kDiag + 16; }

int launch_direct(const double* x, const double* y, const double* z, const double* m, int n, const int* tg, int nt,
                  double eps2, double* gax, double* gay, double* gaz, cudaStream_t s) {
    if (nt <= 0) return MHPC_OK;
    CUDA_TRY(cudaMemsetAsync(gax, 0, sizeof(double) * nt, s));
    CUDA_TRY(cudaMemsetAsync(gay, 0, sizeof(double) * nt, s));
    CUDA_TRY(cudaMemsetAsync(gaz, 0, sizeof(double) * nt, s));
    int bx = (nt + 255) / 256;
    int by = (int)((148L * 8 + bx - 1) / bx);
    if (by < 1) by = 1;
    long maxby = ((long)n + 255) / 256;
    if (by > maxby) by = (int)maxby;
    dim3 grid(bx, by);
    k_direct<<<grid, 256, 0, s>>>(x, y, z, m, n, tg, nt, eps2, gax, gay, gaz);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
