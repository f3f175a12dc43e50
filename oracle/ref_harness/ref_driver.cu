// Reference harness driver: runs milupHPC's own single-rank kernels (compiled
// unmodified from the reference sources, see build_ref.py) on an input file
// and writes their outputs, so that the oracle can be pinned against the
// reference itself.  TEST INFRASTRUCTURE ONLY; built into oracle/_ref/.
//
// The gravity build (Plummer parameter.h) runs: resetArrays,
// computeBoundingBox, buildTree, calculateCentersOfMass (levels 21..1),
// prepareSorting + sortArray (CUB) of keys supplied in the input, and
// computeForces_v2.  The SPH build (Sedov parameter.h) runs: resetArrays,
// computeBoundingBox, buildTree, fixedRadiusNN (v0), calculateDensity,
// calculateSoundSpeed, calculatePressure, internalForces.
// getParticleKeys is not run: it walks child[] past a null slot and reads
// before the start of the array, which is not safe to execute here; keys are
// pinned through the tree instead (every particle's path through the
// reference tree is its key prefix).
//
// Timing: with a third argument K > 0 the driver runs the whole sequence
// above once more untimed, then K more times between CUDA events (gravity
// build: resetArrays, computeBoundingBox, buildTree, calculateCentersOfMass
// 21..1, prepareSorting + sortArray, computeForces_v2; SPH build: resetArrays
// with the noi/nnl memsets, computeBoundingBox, buildTree, fixedRadiusNN,
// calculateDensity, calculateSoundSpeed + calculatePressure, internalForces;
// each reference launch wrapper synchronises the device, as in the reference)
// and prints one line `time_ms <stage> <mean ms>` per stage and for the total.
//
// Input (little-endian binary): int32 n, int32 flags, double theta, double eps2,
// double params[8], then x, y, z, m (n doubles each), then (gravity) keys
// (n uint64) or (SPH) vx, vy, vz, sml, e, p, cs (n doubles each).
// Output: double bbox[6] (min/max x, y, z), int32 tree index (one past the
// last cell), int32 MAX_NUM_INTERACTIONS, then (gravity) sorted[n],
// child[8*numNodes], level, x, y, z, mass [numNodes each], g_ax, g_ay, g_az
// [n each]; (SPH) noi[n], nnl[MAX_NUM_INTERACTIONS*n], rho, cs, p, ax, ay, az,
// drhodt, dedt, dsmldt [n each], double diam, and with BALSARA_SWITCH divv[n],
// curlv[3n] (x, y, z per particle).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "particle_handler.h"
#include "subdomain_key_tree/tree_handler.h"
#include "device_rhs.cuh"
#include "helper.cuh"
#if GRAVITY_SIM
#include "gravity/gravity.cuh"
#endif
#if SPH_SIM
#include "sph/sph.cuh"
#include "sph/density.cuh"
#include "sph/soundspeed.cuh"
#include "sph/pressure.cuh"
#include "sph/internal_forces.cuh"
#include "sph/kernel_handler.cuh"
#include "materials/material_handler.h"
#endif

#include "utils/logger.h"

// the reference defines its logger configuration in main.cpp, which the
// harness does not build; errors only, nothing else printed
structLog LOGCFG = {};

#define CK(x)                                                                   \
    do {                                                                        \
        cudaError_t e_ = (x);                                                   \
        if (e_ != cudaSuccess) {                                                \
            std::fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            std::exit(2);                                                       \
        }                                                                       \
    } while (0)

template <typename T>
static void rd(FILE* f, T* p, size_t n) {
    if (std::fread(p, sizeof(T), n, f) != n) { std::fprintf(stderr, "short input\n"); std::exit(3); }
}
template <typename T>
static void wr(FILE* f, const T* p, size_t n) { std::fwrite(p, sizeof(T), n, f); }
template <typename T>
static std::vector<T> dl(const T* d, size_t n) {
    std::vector<T> h(n);
    CK(cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
}

// Host only, no GPU: `--hilbert in out` converts 21-level Lebesgue keys
// (int32 n, then n uint64) to Hilbert keys with the reference's
// host-callable KeyNS::lebesgue2hilbert(key, MAX_LEVEL, MAX_LEVEL), the
// conversion Tree::getParticleKey applies (tree.cu:233), and writes n uint64.
static int hilbert_keys(const char* in, const char* out) {
    FILE* fi = std::fopen(in, "rb");
    if (!fi) return 1;
    int n = 0;
    rd(fi, &n, 1);
    if (n < 0 || n > (1 << 26)) return 1;
    std::vector<unsigned long long> k(n), h(n);
    rd(fi, k.data(), n);
    std::fclose(fi);
    for (int i = 0; i < n; ++i) h[i] = KeyNS::lebesgue2hilbert((keyType)k[i], MAX_LEVEL, MAX_LEVEL);
    FILE* fo = std::fopen(out, "wb");
    if (!fo) return 1;
    wr(fo, h.data(), n);
    std::fclose(fo);
    std::printf("ok hilbert n=%d\n", n);
    return 0;
}

int main(int argc, char** argv) {
    if (argc == 4 && std::strcmp(argv[1], "--hilbert") == 0) return hilbert_keys(argv[2], argv[3]);
    if (argc != 3 && argc != 4) { std::fprintf(stderr, "usage: %s input output [repeats]\n", argv[0]); return 1; }
    const int repeats = argc == 4 ? std::atoi(argv[3]) : 0;
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi) return 1;
    int n, flags;
    double theta, eps2, par[8];
    rd(fi, &n, 1); rd(fi, &flags, 1); rd(fi, &theta, 1); rd(fi, &eps2, 1); rd(fi, par, 8);
    std::vector<double> x(n), y(n), z(n), m(n);
    rd(fi, x.data(), n); rd(fi, y.data(), n); rd(fi, z.data(), n); rd(fi, m.data(), n);
    // Input conditions the caller (tests/golden/make_golden.py) checks on the
    // CPU before writing the file: n a multiple of 256 in [1024, 65536], or a
    // multiple of 65536 (the reference kernels call __syncthreads inside their
    // per-particle loops, so every thread of a block must run the same number
    // of them: computeForces_v2 strides by its 256 x 256 threads; and
    // computeBoundingBox reads x[0..1023]), pairwise distinct 21-level
    // keys and a shallow tree (buildTree subdivides until two particles
    // separate; computeForces_v2 keeps 128 stack entries per warp without a
    // bound check), fewer than MAX_NUM_INTERACTIONS neighbours per particle
    // (fixedRadiusNN v0 stores without a bound check).
    if (n < 1024 || n % 256 != 0 || (n > 65536 && n % 65536 != 0) || n > (1 << 20)) {
        std::fprintf(stderr, "unsupported n\n");
        return 1;
    }
    const int numNodes = 2 * n + 20000;
    // Every particle array is sized numNodes: fixedRadiusNN v0 reads sml[] at
    // cell indices, which lie past the particle count.
    ParticleHandler ph(numNodes, numNodes);
    TreeHandler th(n, numNodes);
    CK(cudaMemcpy(ph.d_x, x.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_y, y.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_z, z.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_mass, m.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemset(ph.d_nodeType, 0, sizeof(integer) * numNodes));

    // Miluphpc::reset / boundingBox / parallel_tree (src/miluphpc.cpp:679-791, 1088-1182)
    Kernel::Launch::resetArrays(th.d_tree, ph.d_particles, th.d_mutex, n, numNodes, false);
    TreeNS::Kernel::Launch::computeBoundingBox(th.d_tree, ph.d_particles, th.d_mutex, n, 256, false);
    CK(cudaDeviceSynchronize());
    double bb[6];
    CK(cudaMemcpy(&bb[0], th.d_minX, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&bb[1], th.d_maxX, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&bb[2], th.d_minY, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&bb[3], th.d_maxY, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&bb[4], th.d_minZ, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&bb[5], th.d_maxZ, sizeof(double), cudaMemcpyDeviceToHost));
    TreeNS::Kernel::Launch::buildTree(th.d_tree, ph.d_particles, n, n, false);
    CK(cudaDeviceSynchronize());
    int index = 0;
    CK(cudaMemcpy(&index, th.d_index, sizeof(int), cudaMemcpyDeviceToHost));
    if (index <= n || index >= numNodes) { std::fprintf(stderr, "node pool: index %d\n", index); return 4; }

    FILE* fo = std::fopen(argv[2], "wb");
    if (!fo) return 1;
    const int maxnb = MAX_NUM_INTERACTIONS;
    wr(fo, bb, 6);
    wr(fo, &index, 1);
    wr(fo, &maxnb, 1);

#if GRAVITY_SIM
    std::vector<unsigned long long> keys(n);
    rd(fi, keys.data(), n);
    // Miluphpc::parallel_pseudoParticles: calculateCentersOfMass for level 21..1
    for (int level = MAX_LEVEL; level > 0; --level)
        TreeNS::Kernel::Launch::calculateCentersOfMass(th.d_tree, ph.d_particles, n, level, false);
    // presort (src/miluphpc.cpp:2164-2181) with the supplied keys
    keyType *d_keys, *d_keys_out;
    CK(cudaMalloc(&d_keys, sizeof(keyType) * n));
    CK(cudaMalloc(&d_keys_out, sizeof(keyType) * n));
    CK(cudaMemcpy(d_keys, keys.data(), sizeof(keyType) * n, cudaMemcpyHostToDevice));
    TreeNS::Kernel::Launch::prepareSorting(th.d_tree, ph.d_particles, n, n);
    HelperNS::sortArray(th.d_start, th.d_sorted, d_keys, d_keys_out, n);
    const double radius = 0.5 * (bb[1] - bb[0]);
    Gravity::Kernel::Launch::computeForces_v2(th.d_tree, ph.d_particles, radius, n, n, 256, 32, 128, nullptr, theta,
                                             eps2, false);
    CK(cudaDeviceSynchronize());
    wr(fo, dl(th.d_sorted, n).data(), n);
    wr(fo, dl(th.d_child, (size_t)8 * numNodes).data(), (size_t)8 * numNodes);
    wr(fo, dl(ph.d_level, numNodes).data(), numNodes);
    wr(fo, dl(ph.d_x, numNodes).data(), numNodes);
    wr(fo, dl(ph.d_y, numNodes).data(), numNodes);
    wr(fo, dl(ph.d_z, numNodes).data(), numNodes);
    wr(fo, dl(ph.d_mass, numNodes).data(), numNodes);
    wr(fo, dl(ph.d_g_ax, n).data(), n);
    wr(fo, dl(ph.d_g_ay, n).data(), n);
    wr(fo, dl(ph.d_g_az, n).data(), n);
    if (repeats > 0) {
        // stages of one gravity right-hand side, the first pass untimed
        const char* names[6] = {"reset_bbox", "build_tree", "centers_of_mass", "sort", "forces_v2", "total"};
        double acc[6] = {0, 0, 0, 0, 0, 0};
        cudaEvent_t ev[6];
        for (int k = 0; k < 6; ++k) CK(cudaEventCreate(&ev[k]));
        for (int rep = 0; rep <= repeats; ++rep) {
            CK(cudaEventRecord(ev[0]));
            Kernel::Launch::resetArrays(th.d_tree, ph.d_particles, th.d_mutex, n, numNodes, false);
            TreeNS::Kernel::Launch::computeBoundingBox(th.d_tree, ph.d_particles, th.d_mutex, n, 256, false);
            CK(cudaEventRecord(ev[1]));
            TreeNS::Kernel::Launch::buildTree(th.d_tree, ph.d_particles, n, n, false);
            CK(cudaEventRecord(ev[2]));
            for (int level = MAX_LEVEL; level > 0; --level)
                TreeNS::Kernel::Launch::calculateCentersOfMass(th.d_tree, ph.d_particles, n, level, false);
            CK(cudaEventRecord(ev[3]));
            CK(cudaMemcpy(d_keys, keys.data(), sizeof(keyType) * n, cudaMemcpyHostToDevice));
            TreeNS::Kernel::Launch::prepareSorting(th.d_tree, ph.d_particles, n, n);
            HelperNS::sortArray(th.d_start, th.d_sorted, d_keys, d_keys_out, n);
            CK(cudaEventRecord(ev[4]));
            Gravity::Kernel::Launch::computeForces_v2(th.d_tree, ph.d_particles, radius, n, n, 256, 32, 128, nullptr,
                                                     theta, eps2, false);
            CK(cudaEventRecord(ev[5]));
            CK(cudaEventSynchronize(ev[5]));
            int idx2 = 0;
            CK(cudaMemcpy(&idx2, th.d_index, sizeof(int), cudaMemcpyDeviceToHost));
            if (idx2 != index) { std::fprintf(stderr, "tree changed between runs\n"); return 5; }
            if (rep == 0) continue;
            for (int k = 0; k < 5; ++k) {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
                acc[k] += ms;
            }
            float tot = 0.f;
            CK(cudaEventElapsedTime(&tot, ev[0], ev[5]));
            acc[5] += tot;
        }
        for (int k = 0; k < 6; ++k) std::printf("time_ms %s %.6f\n", names[k], acc[k] / repeats);
    }
    cudaFree(d_keys);
    cudaFree(d_keys_out);
#endif

#if SPH_SIM
    std::vector<double> vx(n), vy(n), vz(n), sml(n), e(n), p(n), cs(n);
    rd(fi, vx.data(), n); rd(fi, vy.data(), n); rd(fi, vz.data(), n); rd(fi, sml.data(), n);
    rd(fi, e.data(), n); rd(fi, p.data(), n); rd(fi, cs.data(), n);
    CK(cudaMemcpy(ph.d_vx, vx.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_vy, vy.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_vz, vz.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_sml, sml.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_e, e.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_p, p.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ph.d_cs, cs.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemset(ph.d_materialId, 0, sizeof(integer) * n));
    CK(cudaMemset(ph.d_noi, 0, sizeof(integer) * n));
    CK(cudaMemset(ph.d_nnl, 0xff, sizeof(integer) * (size_t)MAX_NUM_INTERACTIONS * n));
    // material: par = {interactions, alpha, beta, eos type, K, gamma}
    MaterialHandler mh(1, 0, (int)par[0], par[1], par[2]);
    mh.h_materials[0].eos.type = (int)par[3];
    mh.h_materials[0].eos.polytropic_K = par[4];
    mh.h_materials[0].eos.polytropic_gamma = par[5];
    mh.copy(To::device);
    SPH::KernelHandler kh(Smoothing::cubic_spline);
    // Miluphpc::parallel_sph, single rank (src/miluphpc.cpp:2820-2990)
    const double diam = std::abs(bb[1]) + std::abs(bb[0]);
    SPH::Kernel::Launch::fixedRadiusNN(th.d_tree, ph.d_particles, ph.d_nnl, diam, n, n, numNodes);
    SPH::Kernel::Launch::calculateDensity(kh.kernel, th.d_tree, ph.d_particles, ph.d_nnl, n);
    SPH::Kernel::Launch::calculateSoundSpeed(ph.d_particles, mh.d_materials, n);
#if BALSARA_SWITCH
    // src/miluphpc.cpp:2944-2947: divergence and curl of v after the sound speed
    SPH::Kernel::Launch::CalcDivvandCurlv(kh.kernel, ph.d_particles, ph.d_nnl, n);
#endif
    SPH::Kernel::Launch::calculatePressure(mh.d_materials, ph.d_particles, n);
    SPH::Kernel::Launch::internalForces(kh.kernel, mh.d_materials, th.d_tree, ph.d_particles, ph.d_nnl, n);
    CK(cudaDeviceSynchronize());
    wr(fo, dl(ph.d_noi, n).data(), n);
    wr(fo, dl(ph.d_nnl, (size_t)MAX_NUM_INTERACTIONS * n).data(), (size_t)MAX_NUM_INTERACTIONS * n);
    wr(fo, dl(ph.d_rho, n).data(), n);
    wr(fo, dl(ph.d_cs, n).data(), n);
    wr(fo, dl(ph.d_p, n).data(), n);
    wr(fo, dl(ph.d_ax, n).data(), n);
    wr(fo, dl(ph.d_ay, n).data(), n);
    wr(fo, dl(ph.d_az, n).data(), n);
    wr(fo, dl(ph.d_drhodt, n).data(), n);
    wr(fo, dl(ph.d_dedt, n).data(), n);
    wr(fo, dl(ph.d_dsmldt, n).data(), n);
    wr(fo, &diam, 1);
#if BALSARA_SWITCH
    wr(fo, dl(ph.d_divv, n).data(), n);
    wr(fo, dl(ph.d_curlv, (size_t)3 * n).data(), (size_t)3 * n);
#endif
    if (repeats > 0) {
        // stages of one fixed-h SPH right-hand side (Miluphpc::rhs single rank:
        // reset with the neighbour-list memsets, bounding box, tree,
        // parallel_sph), the first pass untimed
        const char* names[7] = {"reset_bbox", "build_tree", "fixed_radius_nn", "density",
                                "sound_speed_pressure", "internal_forces", "total"};
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        cudaEvent_t ev[7];
        for (int k = 0; k < 7; ++k) CK(cudaEventCreate(&ev[k]));
        for (int rep = 0; rep <= repeats; ++rep) {
            CK(cudaEventRecord(ev[0]));
            Kernel::Launch::resetArrays(th.d_tree, ph.d_particles, th.d_mutex, n, numNodes, false);
            CK(cudaMemset(ph.d_noi, 0, sizeof(integer) * n));
            CK(cudaMemset(ph.d_nnl, 0xff, sizeof(integer) * (size_t)MAX_NUM_INTERACTIONS * n));
            TreeNS::Kernel::Launch::computeBoundingBox(th.d_tree, ph.d_particles, th.d_mutex, n, 256, false);
            CK(cudaEventRecord(ev[1]));
            TreeNS::Kernel::Launch::buildTree(th.d_tree, ph.d_particles, n, n, false);
            CK(cudaEventRecord(ev[2]));
            SPH::Kernel::Launch::fixedRadiusNN(th.d_tree, ph.d_particles, ph.d_nnl, diam, n, n, numNodes);
            CK(cudaEventRecord(ev[3]));
            SPH::Kernel::Launch::calculateDensity(kh.kernel, th.d_tree, ph.d_particles, ph.d_nnl, n);
            CK(cudaEventRecord(ev[4]));
            SPH::Kernel::Launch::calculateSoundSpeed(ph.d_particles, mh.d_materials, n);
#if BALSARA_SWITCH
            SPH::Kernel::Launch::CalcDivvandCurlv(kh.kernel, ph.d_particles, ph.d_nnl, n);
#endif
            SPH::Kernel::Launch::calculatePressure(mh.d_materials, ph.d_particles, n);
            CK(cudaEventRecord(ev[5]));
            SPH::Kernel::Launch::internalForces(kh.kernel, mh.d_materials, th.d_tree, ph.d_particles, ph.d_nnl, n);
            CK(cudaEventRecord(ev[6]));
            CK(cudaEventSynchronize(ev[6]));
            int idx2 = 0;
            CK(cudaMemcpy(&idx2, th.d_index, sizeof(int), cudaMemcpyDeviceToHost));
            if (idx2 != index) { std::fprintf(stderr, "tree changed between runs\n"); return 5; }
            if (rep == 0) continue;
            for (int k = 0; k < 6; ++k) {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
                acc[k] += ms;
            }
            float tot = 0.f;
            CK(cudaEventElapsedTime(&tot, ev[0], ev[6]));
            acc[6] += tot;
        }
        for (int k = 0; k < 7; ++k) std::printf("time_ms %s %.6f\n", names[k], acc[k] / repeats);
    }
#endif
    std::fclose(fo);
    std::fclose(fi);
    std::printf("ok n=%d nodes=%d\n", n, index);
    return 0;
}
