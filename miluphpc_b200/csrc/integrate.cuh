#pragma once
#include "common.cuh"

#define MHPC_GATHER_MAX 16

// dst[a][s] = src[a][perm[s]] (gather) or dst[a][perm[s]] = src[a][s] (scatter)
struct GatherList {
    int count;
    const double* src[MHPC_GATHER_MAX];
    double* dst[MHPC_GATHER_MAX];
    const int* isrc;  // optional int array gathered alongside
    int* idst;
    int imax;         // > 0: gathered ints must lie in [0, imax) (material ids); others are
    DevStatus* st;    // reported as MHPC_ERR_ARG (detail: the original index) and clamped
};

int launch_gather(int n, const int* perm, const GatherList& L, cudaStream_t s);
int launch_scatter(int n, const int* perm, const GatherList& L, cudaStream_t s);
int launch_leapfrog_x(const mhpc_particles& p, double dt, cudaStream_t s);
int launch_leapfrog_v(const mhpc_particles& p, double dt, cudaStream_t s);
int launch_euler(const mhpc_particles& p, double dt, int gravity, int sph, int int_rho, int int_e, int int_sml,
                 cudaStream_t s);
int launch_pc_predictor(const mhpc_particles& p, const mhpc_particles& q, const double* dt, int sph, int int_rho,
                        int int_e, cudaStream_t s);
int launch_pc_corrector(const mhpc_particles& p, const mhpc_particles& q, const double* dt, int sph, int int_rho,
                        int int_e, int int_sml, cudaStream_t s);
// part needs 148 * 2 * 6 doubles
int launch_set_time_step(const mhpc_particles& p, int gravity, int sph, double alpha, double beta, int int_rho,
                         double time_left, double dt_max, double* part, double* dt_out, cudaStream_t s);
// Particle removal: keep[i] = 1 for particles inside the criterion's region;
// stable compaction of one array by the exclusive scan (rank) of keep.
int launch_remove_mark(int n, const double* x, const double* y, const double* z, int criterion, double d, int* keep,
                       cudaStream_t s);
int launch_compact_d(int n, const int* keep, const int* rank, const double* src, double* dst, cudaStream_t s);
int launch_compact_i(int n, const int* keep, const int* rank, const int* src, int* dst, cudaStream_t s);
int launch_diagnostics(const mhpc_particles& p, int sph, double* part, double* out, cudaStream_t s);
// Start of a right-hand side: when `fold`, add the finished RHS's counters in
// *st to the run totals (its band counter only when `band`); then zero *st,
// keeping an error code (with its detail and site) when `keep`.
int launch_status_fold(DevStatus* st, RunTotals* run, int fold, int band, int keep, cudaStream_t s);
size_t diagnostics_scratch_doubles();
// W = 1/2 sum m_i phi_i into out[0] (part: diagnostics scratch).
int launch_potential_energy(int n, const double* m, const double* pot, double* part, double* out, cudaStream_t s);
int launch_direct(const double* x, const double* y, const double* z, const double* m, int n, const int* tg, int nt,
                  double eps2, const double* eps2_t, double* gax, double* gay, double* gaz, cudaStream_t s);
