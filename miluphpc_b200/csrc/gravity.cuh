#pragma once
#include "tree.cuh"

struct GravParams {
    int n;
    double eps2;          // global softening eps^2 (config `smoothing`)
    double h_factor;      // softening tied to h: eps_i = h_factor * h_i (0 = off)
    double G;             // gravitational constant (1 unless SI units)
    double theta;         // opening parameter
    const long long* ord; // device bounding box (ordered-int min, max); radius = (max - min) / 2
    double rel_alpha;     // interaction-list walk: relative opening rule with this alpha (0 = off), reading
                          // the previous accelerations from the output arrays before overwriting them
    double quad_alpha;    // relative rule: accepted cells with M l^2 <= quad_alpha |a| d^4 enter as monopoles
    double* pot;          // interaction-list walk: gravitational potential per particle (caller's order),
                          // null = accelerations only
};

// Plain FP64 walk with the reference's computeForces_v2 semantics.
int gravity_v2(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
               const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
               cudaStream_t s);
// Plain FP64 walk with the reference's computeForces_v1 semantics (one walk
// per particle).
int gravity_v1(const TreeDev& T, const GravParams& P, const double* sh, const int* perm, double* gax, double* gay,
               double* gaz, DevStatus* st, cudaStream_t s);
// Mixed FP32 walk, per-lane vote: hi/lo node positions relative to the group
// centre, every particle of the warp votes on each cell, monopole + quadrupole,
// FP64 flush of FP32 partial sums (precision 2).
int gravity_mixed(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
                  const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
                  cudaStream_t s);
// Mixed FP32 walk with interaction lists: lane-parallel traversal against the
// sub-boxes of 64-particle groups, accepted cells and leaves evaluated from
// shared-memory lists (precision 1).
int gravity_lists(const TreeDev& T, const GravParams& P, const double* sx, const double* sy, const double* sz,
                  const double* sh, const int* perm, double* gax, double* gay, double* gaz, DevStatus* st,
                  cudaStream_t s);
