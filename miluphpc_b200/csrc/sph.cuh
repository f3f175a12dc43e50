#pragma once
#include "tree.cuh"

#define MHPC_MAX_MATERIALS 8

struct MatDev {
    int eos_type;
    int interactions;
    double alpha, beta;
    double K, gamma, rho0, bulk, n_exp, shear;
    double cs_init;  // sound speed set by initializeSoundSpeed (Murnaghan, isothermal)
};

struct SphParams {
    int n;
    int maxnb;             // max_num_interactions (list stride per particle)
    int kernel;            // 0 spiky, 1 cubic spline, 2 wendlandc2, 3 wendlandc4, 4 wendlandc6
    int avg_h;             // h_bar = (h_i + h_j)/2 (variable_sml || integrate_sml)
    int integrate_energy;
    int integrate_sml;
    int integrate_density; // density from state (no kernel sum)
    int num_materials;
    int mixed;             // FP32 pair sums on group-relative coordinates
    int balsara;           // Balsara switch on the viscosity (S.bal holds the factors)
    int variable_sml;      // the Balsara gradients use h_bar only under VARIABLE_SML
    const long long* ord;  // device bounding box (ordered-integer min, max): its edge caps h
    MatDev mat[MHPC_MAX_MATERIALS];
};

// Sorted-order views of the SPH state.
struct SphSorted {
    const double *x, *y, *z, *m, *h;
    const double *vx, *vy, *vz, *e;
    const int* mat;        // may be null
    double *rho, *p, *cs;  // sorted outputs of the density/EOS pass (p, cs hold previous values on entry)
    double* bal;           // sorted Balsara factors (written by sph_balsara, read by sph_forces)
    // FP32 pair-sum views (mixed precision), written by sph_density_eos:
    // f0 = (x_hi, y_hi, z_hi, h), f1 = (x_lo, y_lo, z_lo, m) with x = x_hi + x_lo
    // (FP32 split of the FP64 position), f2 = (vx, vy, vz, c_s), f3 = (rho, p/rho^2)
    float4 *f0, *f1, *f2;
    float2* f3;
};

// Squared distance without FMA contraction, summed in the reference's order
// (dx^2 + dy^2) + dz^2: the pair rule's d^2 of every neighbour kernel.
__device__ __forceinline__ double d2_exact(double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Slot k of sorted particle s's neighbour list in the group-transposed layout.
__device__ __forceinline__ size_t nb_index(long s, int k, int maxnb) {
    return ((size_t)(s >> 5) * maxnb + k) * 32 + (s & 31);
}

// Neighbour lists in sorted index space, group-transposed:
// nbr[((s >> 5) * maxnb + k) * 32 + (s & 31)], count noi[s].
int sph_frnn(const TreeDev& T, const SphParams& P, const SphSorted& S, int* nbr, int* noi, DevStatus* st,
             cudaStream_t s);
struct VhBuffers {
    double* hold;        // [n] Jacobi snapshot
    int* done;           // [n] converged (zeroed by the caller before the first sweep)
    int* nit;            // [n] iteration counters (-1 before the first sweep)
    int* count;          // [n] neighbour counts of the last sweep
    int* flags;          // [n] scratch
    int* off;            // [n+1] scratch (scan); off[n] = particles still iterating
    int* list;           // [n] particles still iterating
    void* scan_scratch;
    int* list2;          // [n] second list (list-based form: sweeps after the first alternate lists)
    int* cnt;            // [2] lengths of the alternating lists
};
// Plain variable-h iteration (Jacobi form of fixedRadiusNN_variableSML):
// updates h (sorted, in place) for `sweeps` sweeps; every sweep walks only the
// particles still iterating (compacted list).  Starting h (the caller's h on
// entry) may be the previous step's or a predicted one.
int sph_variable_h(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                   double* h, const VhBuffers& B, int target, int tol, int max_iter, int sweeps, DevStatus* st,
                   cudaStream_t s);
// Density (kernel sum over the lists) + EOS.  P.mixed: the pair sums in FP32 on
// hi/lo-split relative positions with FP64 accumulation (and the FP32 views
// of S filled for sph_forces); otherwise FP64 throughout.
int sph_density_eos(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, const int* perm,
                    double* rho_out, double* p_out, double* cs_out, DevStatus* st, cudaStream_t s);
// Balsara switch (SPH::Kernel::CalcDivvandCurlv, src/sph/kernel.cu:223-342, and
// the factor of internalForces, src/sph/internal_forces.cu:210-217): div v and
// curl v from the neighbour lists, f_i into S.bal; after sph_density_eos.
int sph_balsara(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, DevStatus* st,
                cudaStream_t s);
// Internal forces; P.mixed: pair terms in FP32 from the views sph_density_eos
// filled, FP64 accumulation.
int sph_forces(const SphParams& P, const SphSorted& S, const int* nbr, const int* noi, const int* perm,
               double* ax, double* ay, double* az, double* drhodt, double* dedt, double* dsmldt, DevStatus* st,
               cudaStream_t s);
// Scatter the sorted neighbour lists into the reference layout
// nnl[i * maxnb + k] (original indices) and noi[i].
// particles whose final neighbour count misses |n - target| < tol -> st->sml_out_of_band
int sph_band_stats(const SphParams& P, const int* noi, int target, int tol, DevStatus* st, cudaStream_t s);
int sph_export_nnl(const SphParams& P, const int* nbr, const int* noi, const int* perm, int* nnl, int* noi_out,
                   cudaStream_t s);

// Neighbour-band repair after the variable-h iteration and the list walk (an
// addition of this library; the reference stops at its iteration limit and
// leaves such particles where they are).  `rounds` times: every particle
// whose count misses |n - target| < tol takes, with all other h frozen, the h
// that gives it target + tol - 2 neighbours (from above) or target - tol + 2
// (from below): the midpoint of the two candidate distances around that rank,
// candidates being the j != i with d_ij < h_j within a search radius (h_i
// from above; 1.5 h_i, or 2 h_i below half the wanted count, from below,
// at most twice the h before the first round; the search radius itself when
// it holds too few).  All such particles move
// at once, and the neighbour lists and counts are edited in place pair by
// pair, so they equal a fresh list walk on the new h.
struct BandBuffers {
    int* flags;          // [n] scratch (particles out of the band)
    int* off;            // [n+1] scratch (scan); off[n] = particles out of the band
    int* list;           // [n] particles out of the band
    int* dirty;          // [n] lists with removed entries (zeroed here)
    double* hnew;        // [n] new h (equal to h outside a round)
    double* h0;          // [n] h before the first round
    int2* events;        // [cap_events] pair changes (x >= 0: add (x, y); x < 0: remove (~x, y))
    int cap_events;
    int* ctr;            // [4] events, overflow flag
    void* scan_scratch;
    int* appended;       // [n] lists that received appends (zero outside the calls; cleared by the sort)
};
// Sort the lists marked in `appended` by neighbour index and clear the marks.
int sph_sort_appended(const SphParams& P, int* nbr, const int* noi, int* appended, cudaStream_t s);
int sph_band_fixup(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                   double* h, int* nbr, int* noi, const BandBuffers& B, int target, int tol, int rounds,
                   DevStatus* st, cudaStream_t s);

// The pair changes of moving every particle of `list` from h to hnew, applied
// to the lists and counts in place (events, removals, compaction, appends);
// with `trunc` (variable-h iteration) nothing runs while *trunc is set, and a
// list that would pass maxnb sets it.  ctr[0..1] are reset here; ctr[1]
// reports an event-buffer overflow (no list edited).
int sph_apply_h_changes(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                        const double* h, const double* hnew, int* nbr, int* noi, const int* list,
                        const int* list_count, const BandBuffers& B, int* trunc, DevStatus* st, cudaStream_t s);

// The variable-h iteration of sph_variable_h (the same Jacobi sweeps, the same
// update rule and stopping test) on neighbour lists instead of count walks:
// one list walk with the starting h gives every count of the first sweep;
// after each sweep the pairs changed by the new h are edited into the lists
// (sph_apply_h_changes), so the next sweep's counts are exact without a walk,
// and the lists at the end are those of the final h (the list walk of the
// right-hand side is not needed).  Lists that pass maxnb during the
// iteration, or an event-buffer overflow, fall back to a full list walk after
// that sweep.  Uses B.hnew and B.ctr[0..3]; T.hmax stays an upper bound
// (grow-only) of the current h.
int sph_variable_h_lists(const TreeDev& T, const SphParams& P, const double* x, const double* y, const double* z,
                         double* h, int* nbr, int* noi, const VhBuffers& V, const BandBuffers& B, int target,
                         int tol, int max_iter, int sweeps, DevStatus* st, cudaStream_t s);
