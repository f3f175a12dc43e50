// Reference harness for the integrator update kernels: runs milupHPC's own
// LeapfrogNS::Kernel::updateX / updateV (src/integrator/device_leapfrog.cu:
// 4-58), ExplicitEulerNS::Kernel::update (device_explicit_euler.cu:4-54) and
// PredictorCorrectorEulerNS::Kernel::predictor / corrector
// (device_predictor_corrector_euler.cu:130-300), compiled unmodified from the
// reference sources with the Sedov test case's parameter.h (SPH_SIM 1,
// INTEGRATE_ENERGY 1, INTEGRATE_DENSITY 0, INTEGRATE_SML 1), on a state read
// from a file, and writes the updated arrays.  TEST INFRASTRUCTURE ONLY; built
// into oracle/_ref/ by build_ref.py.
//
// The kernels stride over the particles with no block synchronisation; every
// array they touch is allocated by the reference's own ParticleHandler (with
// initLeapfrog for g_a_old) and IntegratedParticleHandler for n particles.
//
// Input (little-endian): int32 n, double dt, then 26 arrays of n doubles:
// x y z vx vy vz ax ay az g_ax g_ay g_az rho drhodt e dedt sml dsmldt p cs
// (the state), gx2 gy2 gz2 (new g for updateV), pax pay paz (rates of the
// predicted state, with pdedt = dedt / 2 and pdsmldt = dsmldt / 2 formed here
// in FP64 from the state's: exact halvings).
// Output: Euler x y z vx vy vz e sml; leapfrog after updateX x y z g_ax_old
// g_ay_old g_az_old, after updateV vx vy vz; predictor x y z vx vy vz e sml
// cs p; corrector x y z vx vy vz ax ay az e dedt sml dsmldt (n doubles each).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "particle_handler.h"
#include "integrator/device_explicit_euler.cuh"
#include "integrator/device_leapfrog.cuh"
#include "integrator/device_predictor_corrector_euler.cuh"
#include "utils/logger.h"

structLog LOGCFG = {};

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            std::exit(2);                                                                       \
        }                                                                                       \
    } while (0)

static void put(double* d, const std::vector<double>& h) {
    CK(cudaMemcpy(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
}
static void out(FILE* f, const double* d, int n) {
    std::vector<double> h(n);
    CK(cudaMemcpy(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost));
    std::fwrite(h.data(), sizeof(double), n, f);
}

int main(int argc, char** argv) {
    if (argc != 3) { std::fprintf(stderr, "usage: %s input output\n", argv[0]); return 1; }
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi) return 1;
    int n = 0;
    double dt = 0;
    if (std::fread(&n, 4, 1, fi) != 1 || std::fread(&dt, 8, 1, fi) != 1) return 3;
    if (n < 1 || n > (1 << 22)) { std::fprintf(stderr, "unsupported n\n"); return 1; }
    const int kArrays = 26;
    std::vector<std::vector<double>> a(kArrays, std::vector<double>(n));
    for (int k = 0; k < kArrays; ++k)
        if (std::fread(a[k].data(), 8, n, fi) != (size_t)n) { std::fprintf(stderr, "short input\n"); return 3; }
    std::fclose(fi);
    enum { X, Y, Z, VX, VY, VZ, AX, AY, AZ, GX, GY, GZ, RHO, DRHO, E, DE, SML, DSML, P, CS, GX2, GY2, GZ2, PAX,
           PAY, PAZ };
    ParticleHandler ph(n, n);
    ph.initLeapfrog();
    IntegratedParticleHandler ip(n, n);
    auto load = [&]() {
        put(ph.d_x, a[X]); put(ph.d_y, a[Y]); put(ph.d_z, a[Z]);
        put(ph.d_vx, a[VX]); put(ph.d_vy, a[VY]); put(ph.d_vz, a[VZ]);
        put(ph.d_ax, a[AX]); put(ph.d_ay, a[AY]); put(ph.d_az, a[AZ]);
        put(ph.d_g_ax, a[GX]); put(ph.d_g_ay, a[GY]); put(ph.d_g_az, a[GZ]);
        put(ph.d_rho, a[RHO]); put(ph.d_drhodt, a[DRHO]); put(ph.d_e, a[E]); put(ph.d_dedt, a[DE]);
        put(ph.d_sml, a[SML]); put(ph.d_dsmldt, a[DSML]); put(ph.d_p, a[P]); put(ph.d_cs, a[CS]);
    };
    FILE* fo = std::fopen(argv[2], "wb");
    if (!fo) return 1;
    // explicit Euler
    load();
    ExplicitEulerNS::Kernel::Launch::update(ph.d_particles, n, dt);
    out(fo, ph.d_x, n); out(fo, ph.d_y, n); out(fo, ph.d_z, n);
    out(fo, ph.d_vx, n); out(fo, ph.d_vy, n); out(fo, ph.d_vz, n);
    out(fo, ph.d_e, n); out(fo, ph.d_sml, n);
    // leapfrog: drift (g_old = g), new g, kick
    load();
    LeapfrogNS::Kernel::Launch::updateX(ph.d_particles, n, dt);
    out(fo, ph.d_x, n); out(fo, ph.d_y, n); out(fo, ph.d_z, n);
    out(fo, ph.d_g_ax_old, n); out(fo, ph.d_g_ay_old, n); out(fo, ph.d_g_az_old, n);
    put(ph.d_g_ax, a[GX2]); put(ph.d_g_ay, a[GY2]); put(ph.d_g_az, a[GZ2]);
    LeapfrogNS::Kernel::Launch::updateV(ph.d_particles, n, dt);
    out(fo, ph.d_vx, n); out(fo, ph.d_vy, n); out(fo, ph.d_vz, n);
    // predictor-corrector
    load();
    PredictorCorrectorEulerNS::Kernel::Launch::predictor(ph.d_particles, ip.d_integratedParticles, dt, n);
    out(fo, ip.d_x, n); out(fo, ip.d_y, n); out(fo, ip.d_z, n);
    out(fo, ip.d_vx, n); out(fo, ip.d_vy, n); out(fo, ip.d_vz, n);
    out(fo, ip.d_e, n); out(fo, ip.d_sml, n); out(fo, ip.d_cs, n); out(fo, ip.d_p, n);
    // the rates a right-hand side on the predicted state would have written
    std::vector<double> hde(n), hdsml(n);
    for (int i = 0; i < n; ++i) { hde[i] = 0.5 * a[DE][i]; hdsml[i] = 0.5 * a[DSML][i]; }
    put(ip.d_ax, a[PAX]); put(ip.d_ay, a[PAY]); put(ip.d_az, a[PAZ]);
    put(ip.d_dedt, hde); put(ip.d_dsmldt, hdsml); put(ip.d_drhodt, a[DRHO]);
    PredictorCorrectorEulerNS::Kernel::Launch::corrector(ph.d_particles, ip.d_integratedParticles, dt, n);
    out(fo, ph.d_x, n); out(fo, ph.d_y, n); out(fo, ph.d_z, n);
    out(fo, ph.d_vx, n); out(fo, ph.d_vy, n); out(fo, ph.d_vz, n);
    out(fo, ph.d_ax, n); out(fo, ph.d_ay, n); out(fo, ph.d_az, n);
    out(fo, ph.d_e, n); out(fo, ph.d_dedt, n); out(fo, ph.d_sml, n); out(fo, ph.d_dsmldt, n);
    std::fclose(fo);
    CK(cudaDeviceSynchronize());
    std::printf("ok integrators n=%d\n", n);
    return 0;
}
