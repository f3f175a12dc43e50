// FP64 state update, gather/scatter between the caller's particle order and
// the SFC-sorted working order, diagnostics, and FP64 direct summation.
#include "common.cuh"
#include "integrate.cuh"

namespace {

// Every field's load is issued before the first store: the destination
// arrays may alias the sources as far as the compiler knows, so a load after
// a store would wait for the previous load's value (one round trip per field).
__global__ void __launch_bounds__(256) k_gather(int n, const int* __restrict__ perm, GatherList L) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = __ldg(perm + s);
        double v[MHPC_GATHER_MAX];
#pragma unroll
        for (int a = 0; a < MHPC_GATHER_MAX; ++a)
            if (a < L.count) v[a] = __ldg(L.src[a] + o);
#pragma unroll
        for (int a = 0; a < MHPC_GATHER_MAX; ++a)
            if (a < L.count) L.dst[a][s] = v[a];
        if (L.isrc) {
            int v = __ldg(L.isrc + o);
            if (L.imax > 0 && (v < 0 || v >= L.imax)) {
                if (L.st) set_status(L.st, MHPC_ERR_ARG, o);
                v = v < 0 ? 0 : L.imax - 1;
            }
            L.idst[s] = v;
        }
    }
}

__global__ void __launch_bounds__(256) k_scatter(int n, const int* __restrict__ perm, GatherList L) {
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
        const int o = __ldg(perm + s);
        double v[MHPC_GATHER_MAX];
#pragma unroll
        for (int a = 0; a < MHPC_GATHER_MAX; ++a)
            if (a < L.count) v[a] = L.src[a][s];
#pragma unroll
        for (int a = 0; a < MHPC_GATHER_MAX; ++a)
            if (a < L.count) L.dst[a][o] = v[a];
    }
}

// The update kernels round every product and sum separately (__dmul_rn /
// __dadd_rn), in the reference's order of operations, like its -fmad=false
// build: the same inputs give bit-identical states.
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
// a + b * c without contraction
__device__ __forceinline__ double axpy_rn(double a, double b, double c) { return __dadd_rn(a, __dmul_rn(b, c)); }

// LeapfrogNS::Kernel::updateX (src/integrator/device_leapfrog.cu:4-30):
// x += dt (v + 0.5 dt g), g_old = g
__global__ void __launch_bounds__(256) k_leapfrog_x(mhpc_particles p, double dt) {
    const double hdt = mul_rn(0.5, dt);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        const double gx = p.g_ax[i], gy = p.g_ay[i], gz = p.g_az[i];
        p.x[i] = axpy_rn(p.x[i], dt, axpy_rn(p.vx[i], hdt, gx));
        p.y[i] = axpy_rn(p.y[i], dt, axpy_rn(p.vy[i], hdt, gy));
        p.z[i] = axpy_rn(p.z[i], dt, axpy_rn(p.vz[i], hdt, gz));
        p.g_ax_old[i] = gx; p.g_ay_old[i] = gy; p.g_az_old[i] = gz;
    }
}

// LeapfrogNS::Kernel::updateV (device_leapfrog.cu:32-58): v += 0.5 dt (g + g_old)
__global__ void __launch_bounds__(256) k_leapfrog_v(mhpc_particles p, double dt) {
    const double hdt = mul_rn(0.5, dt);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        p.vx[i] = axpy_rn(p.vx[i], hdt, add_rn(p.g_ax[i], p.g_ax_old[i]));
        p.vy[i] = axpy_rn(p.vy[i], hdt, add_rn(p.g_ay[i], p.g_ay_old[i]));
        p.vz[i] = axpy_rn(p.vz[i], hdt, add_rn(p.g_az[i], p.g_az_old[i]));
    }
}

// ExplicitEulerNS::Kernel::update (src/integrator/device_explicit_euler.cu:4-54):
// v += dt (a + g), x += dt v (the new v), rho, e (floored at 1e-50), h
__global__ void __launch_bounds__(256) k_euler(mhpc_particles p, double dt, int gravity, int sph, int int_rho,
                                               int int_e, int int_sml) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        // the reference adds a + g with a zero array for the absent part: 0 + g is exact
        double ax = 0, ay = 0, az = 0;
        if (sph) { ax = p.ax[i]; ay = p.ay[i]; az = p.az[i]; }
        if (gravity) { ax = add_rn(ax, p.g_ax[i]); ay = add_rn(ay, p.g_ay[i]); az = add_rn(az, p.g_az[i]); }
        p.vx[i] = axpy_rn(p.vx[i], dt, ax);
        p.vy[i] = axpy_rn(p.vy[i], dt, ay);
        p.vz[i] = axpy_rn(p.vz[i], dt, az);
        p.x[i] = axpy_rn(p.x[i], dt, p.vx[i]);
        p.y[i] = axpy_rn(p.y[i], dt, p.vy[i]);
        p.z[i] = axpy_rn(p.z[i], dt, p.vz[i]);
        if (int_rho) p.rho[i] = axpy_rn(p.rho[i], dt, p.drhodt[i]);
        if (int_e) {
            p.e[i] = axpy_rn(p.e[i], dt, p.dedt[i]);
            if (p.e[i] < 1e-50) p.e[i] = 1e-50;
        }
        if (int_sml) p.sml[i] = axpy_rn(p.sml[i], dt, p.dsmldt[i]);
    }
}

// PredictorCorrectorEulerNS::Kernel::predictor
// (src/integrator/device_predictor_corrector_euler.cu:206-270): Euler
// prediction of the state into `q` with the step on the device.
__global__ void __launch_bounds__(256) k_pc_predictor(mhpc_particles p, mhpc_particles q, const double* dtp,
                                                      int sph, int int_rho, int int_e) {
    const double dt = *dtp;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        double ax = 0, ay = 0, az = 0;
        if (sph) { ax = p.ax[i]; ay = p.ay[i]; az = p.az[i]; }
        ax = add_rn(ax, p.g_ax[i]); ay = add_rn(ay, p.g_ay[i]); az = add_rn(az, p.g_az[i]);
        q.x[i] = axpy_rn(p.x[i], dt, p.vx[i]);
        q.vx[i] = axpy_rn(p.vx[i], dt, ax);
        q.y[i] = axpy_rn(p.y[i], dt, p.vy[i]);
        q.vy[i] = axpy_rn(p.vy[i], dt, ay);
        q.z[i] = axpy_rn(p.z[i], dt, p.vz[i]);
        q.vz[i] = axpy_rn(p.vz[i], dt, az);
        q.mass[i] = p.mass[i];
        if (sph) {
            if (int_rho) q.rho[i] = axpy_rn(p.rho[i], dt, p.drhodt[i]);
            if (int_e) {
                q.e[i] = axpy_rn(p.e[i], dt, p.dedt[i]);
                if (q.e[i] < 1e-6) q.e[i] = 1e-6;
            } else {
                q.e[i] = p.e[i];
            }
            q.sml[i] = p.sml[i];
            q.cs[i] = p.cs[i];
            q.p[i] = p.p[i];
        }
    }
}

// PredictorCorrectorEulerNS::Kernel::corrector (device_predictor_corrector_euler.cu:130-205)
__global__ void __launch_bounds__(256) k_pc_corrector(mhpc_particles p, mhpc_particles q, const double* dtp,
                                                      int sph, int int_rho, int int_e, int int_sml) {
    const double h = mul_rn(0.5, *dtp);  // dt/2, exact
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        const double pax = sph ? q.ax[i] : 0.0, pay = sph ? q.ay[i] : 0.0, paz = sph ? q.az[i] : 0.0;
        const double cax = sph ? p.ax[i] : 0.0, cay = sph ? p.ay[i] : 0.0, caz = sph ? p.az[i] : 0.0;
        const double gx = p.g_ax[i], gy = p.g_ay[i], gz = p.g_az[i];
        p.x[i] = axpy_rn(p.x[i], h, add_rn(q.vx[i], p.vx[i]));
        p.vx[i] = axpy_rn(p.vx[i], h, add_rn(add_rn(pax, cax), mul_rn(2.0, gx)));
        p.y[i] = axpy_rn(p.y[i], h, add_rn(q.vy[i], p.vy[i]));
        p.vy[i] = axpy_rn(p.vy[i], h, add_rn(add_rn(pay, cay), mul_rn(2.0, gy)));
        p.z[i] = axpy_rn(p.z[i], h, add_rn(q.vz[i], p.vz[i]));
        p.vz[i] = axpy_rn(p.vz[i], h, add_rn(add_rn(paz, caz), mul_rn(2.0, gz)));
        if (sph) {
            p.ax[i] = add_rn(mul_rn(0.5, add_rn(pax, cax)), gx);
            p.ay[i] = add_rn(mul_rn(0.5, add_rn(pay, cay)), gy);
            p.az[i] = add_rn(mul_rn(0.5, add_rn(paz, caz)), gz);
            if (int_rho) {
                p.rho[i] = axpy_rn(p.rho[i], h, add_rn(q.drhodt[i], p.drhodt[i]));
                p.drhodt[i] = mul_rn(0.5, add_rn(q.drhodt[i], p.drhodt[i]));
            }
            if (int_e) {
                p.e[i] = axpy_rn(p.e[i], h, add_rn(q.dedt[i], p.dedt[i]));
                if (p.e[i] < 1e-6) p.e[i] = 1e-6;
                p.dedt[i] = mul_rn(0.5, add_rn(q.dedt[i], p.dedt[i]));
            }
            if (int_sml) {
                p.sml[i] = axpy_rn(p.sml[i], h, add_rn(q.dsmldt[i], p.dsmldt[i]));
                p.dsmldt[i] = mul_rn(0.5, add_rn(q.dsmldt[i], p.dsmldt[i]));
            } else {
                p.sml[i] = q.sml[i];
            }
        }
    }
}

// PredictorCorrectorEulerNS::Kernel::setTimeStep
// (device_predictor_corrector_euler.cu:300-470): per-particle limits
// sqrt(h/|a|) (x 0.2), h/c_s (x 0.4), the viscous Courant limit
// 0.4 h / (c_s + 1.2 (alpha c_s + beta mu_max)) (mu_max is never stored by the
// reference's force kernel, so 0), rho limit for integrated density, and the
// search-radius limit searchRadius / (2 v_max); the reference's final
// cross-block v_max combine takes the minimum of the block maxima, which is
// kept.  Result capped by dt_max and the time left; written to *dt.
struct DtShared {
    double forces, courant, rho, visc, vmax;
};

__global__ void __launch_bounds__(256) k_dt_blocks(mhpc_particles p, int gravity, int sph, double alpha, double beta,
                                                   int int_rho, double* part) {
    double forces = 1.7976931348623157e308, courant = forces, dtrho = forces, visc = forces, vmax = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < p.n; i += (long)gridDim.x * blockDim.x) {
        double ax = 0, ay = 0, az = 0;
        if (gravity) { ax += p.g_ax[i]; ay += p.g_ay[i]; az += p.g_az[i]; }
        if (sph) { ax += p.ax[i]; ay += p.ay[i]; az += p.az[i]; }
        const double h = p.sml[i];
        forces = fmin(forces, sqrt(h / sqrt(ax * ax + ay * ay + az * az)));
        if (sph) {
            const double cs = p.cs[i];
            courant = fmin(courant, h / cs);
            visc = fmin(visc, 0.4 * h / (cs + 1.2 * (alpha * cs + beta * 0.0)));
            if (int_rho && p.drhodt[i] != 0)
                dtrho = fmin(dtrho, 0.1 * (fabs(p.rho[i]) + 0.001) / fabs(p.drhodt[i]));
        }
        vmax = fmax(vmax, sqrt(p.vx[i] * p.vx[i] + p.vy[i] * p.vy[i] + p.vz[i] * p.vz[i]));
    }
    __shared__ double s[5][256];
    s[0][threadIdx.x] = forces; s[1][threadIdx.x] = courant; s[2][threadIdx.x] = dtrho;
    s[3][threadIdx.x] = visc; s[4][threadIdx.x] = vmax;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = fmin(s[k][threadIdx.x], s[k][threadIdx.x + o]);
            s[4][threadIdx.x] = fmax(s[4][threadIdx.x], s[4][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 5) part[blockIdx.x * 5 + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_max_sml(int n, const double* h, double* part);

// search radius from the per-block h maxima, then the final combine
__global__ void k_dt_final_sr(int blocks, const double* hmax_part, const double* part, int int_rho, double time_left,
                              double dt_max, double* dt_out) {
    double hmax = 0.0;
    for (int b = 0; b < blocks; ++b) hmax = fmax(hmax, hmax_part[b]);
    double forces = 1.7976931348623157e308, courant = forces, dtrho = forces, visc = forces, vmax = 0.0;
    for (int b = 0; b < blocks; ++b) {
        forces = fmin(forces, part[5 * b]);
        courant = fmin(courant, part[5 * b + 1]);
        dtrho = fmin(dtrho, part[5 * b + 2]);
        visc = fmin(visc, part[5 * b + 3]);
        vmax = b == 0 ? part[5 * b + 4] : fmin(vmax, part[5 * b + 4]);
    }
    const double search_radius = 2.0 * hmax;
    double dt = fmin(0.4 * courant, 0.2 * forces);
    if (vmax > 0. && search_radius > 0.) dt = fmin(dt, search_radius / (2 * vmax));
    if (int_rho) dt = fmin(dt, dtrho);
    dt = fmin(dt, visc);
    dt = fmin(dt, time_left);
    if (dt > dt_max) dt = dt_max;
    *dt_out = dt;
}

__global__ void k_max_sml(int n, const double* h, double* part) {
    double m = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) m = fmax(m, h[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(MHPC_FULL, m, o));
    __shared__ double s[8];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < 8; ++k) m = fmax(m, s[k]);
        part[blockIdx.x] = m;
    }
}

// 0 kinetic energy, 1 internal energy, 2-4 momentum, 5-7 angular momentum,
// 8-10 mass-weighted position sums, 11 total mass
constexpr int kDiag = 12;

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
        acc[11] += m;
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

// block sums in block order (deterministic); the centre of mass is the
// mass-weighted position sum over the total mass
__global__ void k_diag_final(int blocks, const double* part, double* out) {
    __shared__ double tot[kDiag];
    if (threadIdx.x < kDiag) {
        double v = 0;
        for (int b = 0; b < blocks; ++b) v += part[b * kDiag + threadIdx.x];
        tot[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDiag) {
        const double v = tot[threadIdx.x];
        out[threadIdx.x] = (threadIdx.x >= 8 && threadIdx.x < 11) ? (tot[11] > 0 ? v / tot[11] : 0.0) : v;
    }
}

// Direct summation: blockIdx.x covers 256 targets (one per thread), blockIdx.y
// a slice of the sources, staged 256 at a time in shared memory.
__global__ void __launch_bounds__(256) k_direct(const double* __restrict__ x, const double* __restrict__ y,
                                                const double* __restrict__ z, const double* __restrict__ m, int n,
                                                const int* __restrict__ tg, int nt, double eps2,
                                                const double* __restrict__ eps2_t, double* gax, double* gay,
                                                double* gaz) {
    __shared__ double4 src[256];
    const int t = blockIdx.x * 256 + threadIdx.x;
    const bool valid = t < nt;
    const int ti = valid ? tg[t] : 0;
    const double px = x[ti], py = y[ti], pz = z[ti];
    if (eps2_t && valid) eps2 += eps2_t[t];  // softening of the target (h-tied rule)
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

// FP32 FMA throughput probe on the paired instruction the gravity walk
// issues (FFMA2: two FP32 fused multiply-adds per lane): 8 independent
// chains of float2 per thread, i.e. 16 FP32 FMAs per iteration.
constexpr int kFmaIters = 2048;
__global__ void __launch_bounds__(256) k_fma_peak(float* out, float b, float c) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = make_float2(threadIdx.x * 1e-3f + k, threadIdx.x * 2e-3f - k);
    const float2 B = make_float2(b, b), C = make_float2(c, c);
    for (int i = 0; i < kFmaIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = __ffma2_rn(a[k], B, C);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
    if (s == 1234.5f) out[blockIdx.x] = s;
}

// ------------------------------------------------------ particle removal
// ParticlesNS::Kernel::mark2remove with applySphericalCriterion /
// applyCubicCriterion (src/subdomain_key_tree/subdomain.cu:2161-2240): a
// particle is kept when sqrt(x^2 + y^2 + z^2) < d (criterion 0) or when
// |x|, |y|, |z| < d (criterion 1); products and sums explicitly rounded like
// the reference's -fmad=false build.
__global__ void __launch_bounds__(256) k_remove_mark(int n, const double* __restrict__ x,
                                                     const double* __restrict__ y, const double* __restrict__ z,
                                                     int criterion, double d, int* keep) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double xi = x[i], yi = y[i], zi = z[i];
        bool k;
        if (criterion == 0)
            k = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(xi, xi), __dmul_rn(yi, yi)), __dmul_rn(zi, zi))) < d;
        else
            k = fabs(xi) < d && fabs(yi) < d && fabs(zi) < d;
        keep[i] = k ? 1 : 0;
    }
}

// Stable compaction of one array: kept entries move to their rank among the
// kept ones (the reference's stable sort by the removal flag).
template <typename T>
__global__ void __launch_bounds__(256) k_compact_field(int n, const int* __restrict__ keep,
                                                       const int* __restrict__ rank, const T* __restrict__ src,
                                                       T* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (keep[i]) dst[rank[i]] = src[i];
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
    const double flops = 2.0 * 16 * kFmaIters * 256.0 * blocks * reps;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cudaGetLastError() == cudaSuccess ? MHPC_OK : MHPC_ERR_CUDA;
}

__global__ void k_status_fold(DevStatus* st, RunTotals* run, int fold, int band, int keep) {
    // keep: an error of a right-hand side the host has not read yet stays
    // (code, detail, site), so that the kernels of the next one skip and the
    // host sees the first error when it reads the status
    const int code = st->code, detail = st->detail, site = st->timeout_site;
    if (fold && threadIdx.x == 0) {
        const unsigned long long oob = (unsigned long long)max(st->sml_out_of_band, 0);
        run->rhs += 1;
        run->oob_sum += oob;
        run->oob_max = oob > run->oob_max ? oob : run->oob_max;
        if (band && st->sml_band_before >= 0) {
            run->before_sum += (unsigned long long)st->sml_band_before;
            run->band_rhs += 1;
        }
        run->used_sum += (unsigned long long)max(st->predictor_used, 0);
        run->fallback_sum += (unsigned long long)max(st->predictor_fallback, 0);
    }
    __syncthreads();
    int* w = reinterpret_cast<int*>(st);
    for (int i = threadIdx.x; i < (int)(sizeof(DevStatus) / sizeof(int)); i += blockDim.x) w[i] = 0;
    __syncthreads();
    if (keep && code && threadIdx.x == 0) {
        st->code = code;
        st->detail = detail;
        st->timeout_site = site;
    }
}

int launch_status_fold(DevStatus* st, RunTotals* run, int fold, int band, int keep, cudaStream_t s) {
    k_status_fold<<<1, 32, 0, s>>>(st, run, fold, band, keep);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
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

int launch_pc_predictor(const mhpc_particles& p, const mhpc_particles& q, const double* dt, int sph, int int_rho,
                        int int_e, cudaStream_t s) {
    k_pc_predictor<<<grid_for(p.n, 256, 148 * 16), 256, 0, s>>>(p, q, dt, sph, int_rho, int_e);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_pc_corrector(const mhpc_particles& p, const mhpc_particles& q, const double* dt, int sph, int int_rho,
                        int int_e, int int_sml, cudaStream_t s) {
    k_pc_corrector<<<grid_for(p.n, 256, 148 * 16), 256, 0, s>>>(p, q, dt, sph, int_rho, int_e, int_sml);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_set_time_step(const mhpc_particles& p, int gravity, int sph, double alpha, double beta, int int_rho,
                         double time_left, double dt_max, double* part, double* dt_out, cudaStream_t s) {
    const int blocks = 148 * 2;
    // search radius = 2 max(h) (Miluphpc::parallel_sph, src/miluphpc.cpp:2430-2433)
    k_max_sml<<<blocks, 256, 0, s>>>(p.n, p.sml, part);
    k_dt_blocks<<<blocks, 256, 0, s>>>(p, gravity, sph, alpha, beta, int_rho, part + blocks);
    k_dt_final_sr<<<1, 1, 0, s>>>(blocks, part, part + blocks, int_rho, time_left, dt_max, dt_out);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_diagnostics(const mhpc_particles& p, int sph, double* part, double* out, cudaStream_t s) {
    const int blocks = 148 * 4;
    k_diag<<<blocks, 256, 0, s>>>(p, sph, part);
    k_diag_final<<<1, 32, 0, s>>>(blocks, part, out);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

size_t diagnostics_scratch_doubles() { return 148 * 4 * kDiag + 16; }

namespace {
// W = 1/2 sum m_i phi_i: per-block partial sums, then one block adds them in
// block order (deterministic)
__global__ void __launch_bounds__(256) k_pot_part(int n, const double* __restrict__ m,
                                                  const double* __restrict__ pot, double* part) {
    double acc = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        acc += 0.5 * m[i] * pot[i];
    __shared__ double sh[8];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MHPC_FULL, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < 8; ++q) v += sh[q];
        part[blockIdx.x] = v;
    }
}

__global__ void k_pot_final(int blocks, const double* part, double* out) {
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += part[b];
    out[0] = v;
}
}  // namespace

int launch_potential_energy(int n, const double* m, const double* pot, double* part, double* out, cudaStream_t s) {
    const int blocks = 148 * 4;
    k_pot_part<<<blocks, 256, 0, s>>>(n, m, pot, part);
    k_pot_final<<<1, 1, 0, s>>>(blocks, part, out);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_direct(const double* x, const double* y, const double* z, const double* m, int n, const int* tg, int nt,
                  double eps2, const double* eps2_t, double* gax, double* gay, double* gaz, cudaStream_t s) {
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
    k_direct<<<grid, 256, 0, s>>>(x, y, z, m, n, tg, nt, eps2, eps2_t, gax, gay, gaz);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_remove_mark(int n, const double* x, const double* y, const double* z, int criterion, double d, int* keep,
                       cudaStream_t s) {
    k_remove_mark<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, x, y, z, criterion, d, keep);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_compact_d(int n, const int* keep, const int* rank, const double* src, double* dst, cudaStream_t s) {
    k_compact_field<double><<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, keep, rank, src, dst);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}

int launch_compact_i(int n, const int* keep, const int* rank, const int* src, int* dst, cudaStream_t s) {
    k_compact_field<int><<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, keep, rank, src, dst);
    CUDA_TRY(cudaGetLastError());
    return MHPC_OK;
}
