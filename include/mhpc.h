/*
 * mhpc.h — C ABI of the B200-native right-hand side of milupHPC.
 *
 * The library replaces the single-rank path of Miluphpc::rhs()
 * (include/miluphpc.h:478, src/miluphpc.cpp:387-562 of milupHPC) and the
 * integrator kernels that call it.  Every entry point takes plain pointers and
 * sizes; device pointers are CUDA device addresses, `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  All
 * functions return an mhpc status code (MHPC_OK = 0) and never abort the
 * process or trap the GPU.  Work is stream-ordered; functions that must read
 * a device result on the host (status words, counters) synchronise `stream`
 * and say so.
 */
#ifndef MHPC_H
#define MHPC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
/* Replaces host exit(1) (src/miluphpc.cpp:974-981), device assert(0)
 * (include/cuda_utils/cuda_utilities.cuh:41-73) and gpuErrorcheck aborts. */
enum mhpc_status {
    MHPC_OK = 0,
    MHPC_ERR_ARG = 1,         /* null pointer, negative size, bad enum */
    MHPC_ERR_CUDA = 2,        /* CUDA runtime error (launch, copy, alloc) */
    MHPC_ERR_CAPACITY = 3,    /* n larger than the context's capacity */
    MHPC_ERR_NODE_POOL = 4,   /* tree cells exceed the node pool */
    MHPC_ERR_DEPTH = 5,       /* a traversal exceeded its depth / stack bound */
    MHPC_ERR_NEIGHBOURS = 6,  /* a particle has more than max_num_interactions */
    MHPC_ERR_NAN = 7,         /* non-finite position or non-positive density */
    MHPC_ERR_CONFIG = 8,      /* .info / .cfg file missing or malformed */
    MHPC_ERR_NO_DEVICE = 9,   /* no CUDA device */
    MHPC_ERR_TIMEOUT = 10,    /* a bounded device-side wait ran out */
    MHPC_ERR_UNSUPPORTED = 11 /* option not implemented in this build */
};

const char* mhpc_status_string(int status);
int mhpc_version(void);

/* ------------------------------------------------------------ parameters */
/* Run-time form of SimulationParameters (include/parameter.h:122-159) plus
 * the compile-time physics switches of include/parameter.h:25-108, which are
 * run-time flags here. */
typedef struct mhpc_config {
    /* .info keys (src/main.cpp:165-237) */
    int integrator;            /* 0 explicit Euler, 1 predictor-corrector Euler, 2 leapfrog */
    double time_step;
    double max_time_step;
    double time_end;
    int sfc;                   /* 0 Lebesgue, 1 Hilbert */
    double theta;              /* Barnes-Hut opening parameter (squared-ratio form of v2) */
    double smoothing;          /* gravitational softening eps^2, added to r^2 */
    int smoothing_kernel;      /* 0 spiky, 1 cubic spline, 2 wendlandc2, 3 wendlandc4, 4 wendlandc6 */
    int gravity_force_version; /* 0 warp-voted walk (computeForces_v2), 2 per-particle (computeForces_v1) */
    int sph_frnn_version;      /* 0 (fixedRadiusNN) */
    int calculate_energy;
    int calculate_angular_momentum;
    int calculate_center_of_mass;
    int remove_particles;
    int remove_particles_criterion;
    double remove_particles_dimension;
    /* parameter.h switches */
    int gravity;               /* GRAVITY_SIM */
    int sph;                   /* SPH_SIM */
    int integrate_energy;      /* INTEGRATE_ENERGY */
    int integrate_density;     /* INTEGRATE_DENSITY */
    int integrate_sml;         /* INTEGRATE_SML */
    int variable_sml;          /* VARIABLE_SML */
    int si_units;              /* SI_UNITS (G = 6.67430e-11 when set) */
    int max_num_interactions;  /* MAX_NUM_INTERACTIONS (180) */
    int nb_tolerance;          /* TOLERANCE_WANTED_NUMBER_OF_INTERACTIONS (5) */
    int max_sml_iterations;    /* MAX_VARIABLE_SML_ITERATIONS (5) */
    /* additions of this library */
    int precision;             /* 0 plain FP64 (reference semantics); mixed FP32 split + quadrupoles:
                                  1 interaction lists (sub-box criterion), 2 per-lane vote */
    double theta_mixed;        /* opening parameter of the mixed walk (same squared-ratio meaning) */
    int learned_h;             /* 1: MLP smoothing-length predictor with plain fallback */
    int softening_mode;        /* 0 global eps^2, 1 eps_i = softening_h_factor * h_i (plus eps^2) */
    double softening_h_factor;
    double node_pool_factor;   /* tree cell pool = node_pool_factor * capacity + 20000 */
    int gravity_mac;           /* mixed walk (precision 1) opening rule: 0 geometric (theta_mixed); 1
                                  relative: a cell of mass M, edge l is accepted for a group only if
                                  d >= l and M l^3 <= mac_alpha |a| d^5 (d: distance from the cell's
                                  centre of mass to the group, |a|: the group's smallest acceleration of
                                  the previous right-hand side, found in g_ax/g_ay/g_az when the walk
                                  starts); the first gravity call on a context uses the geometric rule */
    double mac_alpha;          /* accuracy parameter of the relative rule (0.003: p99 force error ~8e-4) */
    int balsara;               /* BALSARA_SWITCH: viscous mu_ij scaled by (f_i + f_j)/2,
                                  f = |div v| / (|div v| + |curl v| + 1e-4 c_s / h) */
    double mac_quad_alpha;     /* relative rule only: an accepted cell whose quadrupole term is small,
                                  M l^2 <= mac_quad_alpha |a| d^4 for every sub-box, enters as a monopole
                                  (0: every accepted cell with its quadrupole) */
    int sml_band_rounds;       /* variable h: rounds of the neighbour-band repair after the reference's
                                  iteration (0: none, the reference's behaviour).  Each round, every
                                  particle whose final count misses |n - target| < tol takes, with the
                                  other h frozen, the h giving it target + tol - 2 (from above) or
                                  target - tol + 2 (from below) neighbours; lists and counts are updated
                                  pair by pair.  Not in the reference. */
    int learned_refresh_every; /* learned h, once trained: every this many right-hand sides the
                                  predictor takes learned_refresh_iters Adam steps on the (features,
                                  converged h) pairs collected so far, on the library's stream with
                                  no host synchronisation, so that it follows the flow as it evolves
                                  (0: never; default 10) */
    int learned_refresh_iters; /* Adam steps (mini-batches of 8192 pairs, rate 1e-3) per refresh
                                  (default 32) */
} mhpc_config;

/* Material (include/materials/material.cuh:123-150), one entry of the
 * materials list of a .cfg file. */
typedef struct mhpc_material {
    int id;
    int interactions;          /* variable-h target neighbour count */
    double sml;                /* initial smoothing length = kernel support radius */
    double alpha, beta;        /* artificial_viscosity */
    int eos_type;              /* 0 polytropic, 1 Murnaghan, 3 isothermal, 9 ideal gas, 12 locally isothermal */
    double polytropic_K, polytropic_gamma, rho_0, bulk_modulus, n, shear_modulus;
} mhpc_material;

void mhpc_config_default(mhpc_config* cfg);
/* ConfigParser + src/main.cpp:165-237: read a .info (Boost property-tree
 * INFO syntax: `key value`, `;` comments, `{}` blocks ignored) file. */
int mhpc_config_from_info(const char* path, mhpc_config* cfg);
/* MaterialHandler(const char*) (src/materials/material_handler.cpp:58-150):
 * read a libconfig `materials = ( {...}, ... );` file.  Writes at most `cap`
 * entries indexed by ID and the number found to *count. */
int mhpc_materials_from_cfg(const char* path, mhpc_material* out, int cap, int* count);

/* ------------------------------------------------------------- particles */
/* Mirror of the Particles SoA (include/particles.cuh; allocation
 * src/particle_handler.cpp:8-60,148-170).  Device pointers, FP64 state.
 * x, y, z, mass have num_nodes entries; when num_nodes >= n + cells the
 * cells' centres of mass are written after the particles, as in the
 * reference.  Pointers marked optional may be NULL. */
typedef struct mhpc_particles {
    int n;                     /* numParticlesLocal */
    int num_nodes;             /* length of x, y, z, mass (>= n) */
    double *x, *y, *z, *mass;
    double *vx, *vy, *vz;
    double *ax, *ay, *az;              /* SPH acceleration */
    double *g_ax, *g_ay, *g_az;        /* gravitational acceleration */
    double *g_ax_old, *g_ay_old, *g_az_old; /* leapfrog only */
    double *sml, *rho, *p, *cs, *e;
    double *drhodt, *dedt, *dsmldt;
    int *noi;                  /* optional: neighbour counts */
    int *nnl;                  /* optional: n * max_num_interactions neighbour list (original indices) */
    int *material_id;          /* optional: NULL = material 0 for all */
    int *level;                /* optional: num_nodes tree levels */
} mhpc_particles;

/* ------------------------------------------------ stateless building blocks */
/* TreeNS::Kernel::computeBoundingBox (src/subdomain_key_tree/tree.cu:302-437)
 * after Kernel::resetArrays (src/device_rhs.cu:24-33): cubic box that always
 * contains the origin.  bbox_dev receives 6 doubles {minX,maxX,minY,maxY,
 * minZ,maxZ} in device memory. */
int mhpc_bbox(const double* x, const double* y, const double* z, int n, double* bbox_dev,
              void* stream);
/* SubDomainKeyTreeNS::Kernel::getParticleKeys (src/subdomain_key_tree/
 * subdomain.cu:849-894) / Tree::getParticleKey (tree.cu:157-240): 21-level
 * Lebesgue (curve 0) or Hilbert (curve 1) keys from a device bbox. */
int mhpc_keys(const double* x, const double* y, const double* z, int n, const double* bbox_dev,
              int curve, uint64_t* keys, void* stream);
/* HelperNS::sortArray (src/helper.cu:150-166) with TreeNS::prepareSorting
 * (tree.cu:1404-1413): stable ascending sort of 64-bit keys with int values
 * (vals_in NULL = 0..n-1).  Scratch is caller-provided device memory of
 * mhpc_sort_scratch_bytes(n) bytes; the inputs are not modified. */
size_t mhpc_sort_scratch_bytes(int n);
int mhpc_sort_pairs(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out,
                    int* vals_out, int n, void* scratch, size_t scratch_bytes, void* stream);

/* Sort without any device allocation.  No counterpart in the reference (its
 * sortArray allocates temporary storage on every call).  For callers that
 * cannot allocate device memory — applications whose own memory pool has
 * reserved the GPU at start-up, so a cudaMalloc fails or fragments it, and
 * services that forbid allocation after initialisation — this variant of
 * mhpc_sort_pairs keeps its scratch in a fixed device array inside the
 * library, sized for at most mhpc_sort_noalloc_max_n() (= 1048576) keys
 * (about 16 MB, held on every GPU that loads the library until the process
 * exits).  Larger n returns MHPC_ERR_CAPACITY.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  The address is
 * kept for the life of the process: after cudaDeviceReset (or anything else
 * that destroys and recreates the device's primary context) the library's
 * module may load at another address, so do not call this entry point on that
 * device again in the same process.  All calls share
 * the one array, so calls whose work overlaps on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  status_dev
 * (optional, device int) receives MHPC_OK or MHPC_ERR_TIMEOUT in stream order.
 * The caller still owns keys/values in and out; nothing is allocated or
 * freed. */
int mhpc_sort_noalloc_max_n(void);
int mhpc_sort_pairs_noalloc(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out,
                            int* vals_out, int n, int* status_dev, void* stream);

/* ------------------------------------------------------------ the context */
typedef struct mhpc_ctx mhpc_ctx;

/* Allocates every workspace buffer for up to `capacity` particles once
 * (replaces the handlers' cudaMalloc, src/particle_handler.cpp:148+ and
 * src/subdomain_key_tree/tree_handler.cpp:6-36).  No call below allocates
 * device memory, with two stated exceptions: mhpc_integrate_host allocates its
 * two device mirrors of the state on its first call, and mhpc_fp32_peak allocates
 * and frees a small buffer.  A gravity context also holds 4 * capacity
 * doubles for mhpc_potential. */
int mhpc_ctx_create(mhpc_ctx** out, int capacity, const mhpc_config* cfg,
                    const mhpc_material* materials, int num_materials);
int mhpc_ctx_destroy(mhpc_ctx* ctx);
int mhpc_ctx_set_stream(mhpc_ctx* ctx, void* stream);
int mhpc_ctx_set_config(mhpc_ctx* ctx, const mhpc_config* cfg);

/* Miluphpc::rhs(step, selfGravity, assignParticlesToProcess)
 * (include/miluphpc.h:478, src/miluphpc.cpp:387-562) on one GPU: bbox, keys,
 * sort, tree, centres of mass, gravity (if cfg->gravity && self_gravity),
 * SPH neighbour search, density, sound speed, pressure and internal forces
 * (if cfg->sph).  Results land in the SoA.  Runs on `stream`, which becomes
 * the context's stream (as mhpc_ctx_set_stream).  Synchronises the stream
 * once at the end to read the device status word; *ms_out (optional)
 * receives the device time of the call (the reference's rhs() returns the
 * summed kernel milliseconds). */
int mhpc_rhs(mhpc_ctx* ctx, const mhpc_particles* p, int step, int self_gravity, void* stream, float* ms_out);
/* Same without the final synchronisation: the status is read by
 * mhpc_ctx_status().  Capturable into a CUDA graph.  A right-hand side that
 * starts before the host has read the status of the previous one keeps that
 * one's error code (its kernels then do nothing), so the first error of a
 * queued sequence is the one reported. */
int mhpc_rhs_async(mhpc_ctx* ctx, const mhpc_particles* p, int step, int self_gravity);
int mhpc_ctx_status(mhpc_ctx* ctx);

/* One integrator step (src/integrator/leapfrog.cpp:21-117,
 * explicit_euler.cpp:17-99, predictor_corrector_euler.cpp:47-151) with the
 * integrator of cfg: calls the RHS and the FP64 update kernels.  step 0 runs
 * the extra initial RHS of the leapfrog.  dt_out (optional) receives the
 * step size used. */
int mhpc_integrate(mhpc_ctx* ctx, const mhpc_particles* p, int step, double* dt_out);
/* The same step with HOST (pinned or pageable) state arrays: copies the state
 * in, runs the step, copies the state and accelerations out.  Uses one of the
 * context's two device mirrors (allocated on first use, each the state fields
 * of `capacity` particles).  Returns when the results are in the host arrays
 * (mhpc_integrate_host_async + mhpc_host_wait). */
int mhpc_integrate_host(mhpc_ctx* ctx, mhpc_particles* host, int step, double* dt_out);
/* The host-state step without waiting (the leapfrog's step 0 and the
 * predictor-corrector read a device value and wait for it): successive calls
 * use the two device mirrors in turn; every field is copied in as soon as its
 * mirror is free and the previous step's copy-out of that field has landed
 * (the host arrays are read and written in place), and copied out after the
 * compute, velocities first.  So one step's masses and (leapfrog) drifted
 * positions go in while the previous step computes, and its other fields as
 * soon as the previous step's copies of them are out.  The host arrays must
 * not be read or written until mhpc_host_wait returns; an error of any queued
 * step is reported there. */
int mhpc_integrate_host_async(mhpc_ctx* ctx, mhpc_particles* host, int step, double* dt_out);
/* Wait until every copy of the host-state steps issued so far has finished;
 * returns the device status. */
int mhpc_host_wait(mhpc_ctx* ctx);

/* Sub-stages, one per group of the reference's Launch:: wrappers (which
 * take the device Tree / Particles and return kernel milliseconds after a
 * device synchronisation, include/cuda_utils/cuda_launcher.cuh:114-141).
 * Here each is stream-ordered on the context's stream with no
 * synchronisation; the status word is read by mhpc_ctx_status().  Called in
 * the order below they make up mhpc_rhs_async; a call whose inputs the
 * previous stages did not produce for this particle count returns
 * MHPC_ERR_ARG.  mhpc_bbox, mhpc_keys and mhpc_sort_pairs above are the
 * stateless forms of the first three steps. */
/* bbox (TreeNS::computeBoundingBox, tree.cu:302-437), keys (getParticleKeys,
 * subdomain.cu:849-894), sort (sortArray, helper.cu:150-166), gather into
 * SFC order, and the octree (TreeNS::buildTree, tree.cu:768-1082); resets the
 * status word as the start of a right-hand side. */
int mhpc_tree_build(mhpc_ctx* ctx, const mhpc_particles* p);
/* TreeNS::calculateCentersOfMass (tree.cu:1416-1497, all levels), with the
 * mixed walks' quadrupoles and node records (gravity contexts whose
 * precision is >= 1) and the node boxes / largest h below each node (SPH). */
int mhpc_com(mhpc_ctx* ctx, const mhpc_particles* p);
/* Gravity::computeForces_v2 / _v1 (gravity.cu:726-903 / 252-396) or the
 * mixed walk: precision -1 the configured one, 0 plain FP64
 * (gravity_force_version selects v2 or v1), 1 interaction lists, 2 per-lane
 * vote; 1 and 2 need a context whose configured precision is >= 1. */
int mhpc_gravity(mhpc_ctx* ctx, const mhpc_particles* p, int precision);
/* SPH::fixedRadiusNN_variableSML (sph.cu:739-961, Jacobi form) when
 * variable_h, started from the learned prediction when predictor (the
 * context needs cfg->learned_h), then SPH::fixedRadiusNN (sph.cu:93-281). */
int mhpc_frnn(mhpc_ctx* ctx, const mhpc_particles* p, int variable_h, int predictor);
/* calculateDensity (density.cu:8-72), calculateSoundSpeed (soundspeed.cu:
 * 38-97), calculatePressure (pressure.cu:5-87), and the Balsara factors
 * (kernel.cu:223-342) when configured. */
int mhpc_density_eos(mhpc_ctx* ctx, const mhpc_particles* p);
/* SPH::Kernel::internalForces (internal_forces.cu:4-668); also writes nnl /
 * noi when the SoA has them, the band statistic, and the learned features. */
int mhpc_forces(mhpc_ctx* ctx, const mhpc_particles* p);
/* Coarser groupings of the same stages. */
int mhpc_stage_tree(mhpc_ctx* ctx, const mhpc_particles* p);    /* mhpc_tree_build + mhpc_com */
int mhpc_stage_gravity(mhpc_ctx* ctx, const mhpc_particles* p); /* mhpc_gravity(ctx, p, -1) */
int mhpc_stage_sph(mhpc_ctx* ctx, const mhpc_particles* p);     /* frnn + density_eos + forces as configured */

/* Integrator update kernels alone (no right-hand side), FP64, stream-ordered
 * on the context's stream, with the context's physics switches.
 * half 0: LeapfrogNS::Kernel::updateX (device_leapfrog.cu:4-30), drift and
 * g_a_old = g_a; half 1: updateV (device_leapfrog.cu:32-58), kick with the
 * mean of g_a and g_a_old. */
int mhpc_integrate_leapfrog(mhpc_ctx* ctx, const mhpc_particles* p, double dt, int half);
/* ExplicitEulerNS::Kernel::update (device_explicit_euler.cu:4-54). */
int mhpc_integrate_euler(mhpc_ctx* ctx, const mhpc_particles* p, double dt);
/* PredictorCorrectorEulerNS::Kernel::setTimeStep (device_predictor_corrector_
 * euler.cu:300-470): the step size, capped by max_time_step and time_left,
 * into *dt_dev (device).  Reads g_a (gravity), a, c_s, rho, drho/dt (SPH),
 * h and v of every particle. */
int mhpc_integrate_pc_step_size(mhpc_ctx* ctx, const mhpc_particles* p, double time_left, double* dt_dev);
/* PredictorCorrectorEulerNS::Kernel::predictor (device_predictor_corrector_
 * euler.cu:206-270): the Euler-predicted state of p into q (the reference's
 * IntegratedParticles) with the step *dt_dev; g_a is read (zero arrays
 * without gravity, as in the reference). */
int mhpc_integrate_pc_predictor(mhpc_ctx* ctx, const mhpc_particles* p, const mhpc_particles* q,
                                const double* dt_dev);
/* PredictorCorrectorEulerNS::Kernel::corrector (device_predictor_corrector_
 * euler.cu:130-205): p advanced with the mean of its rates and those of q
 * (the right-hand side evaluated on q). */
int mhpc_integrate_pc_corrector(mhpc_ctx* ctx, const mhpc_particles* p, const mhpc_particles* q,
                                const double* dt_dev);

/* Parity exports (synchronise the stream). */
/* Sorted keys and the permutation tree->sorted (device pointers, n entries). */
int mhpc_export_sorted(mhpc_ctx* ctx, uint64_t* keys_dev, int* perm_dev);
/* Tree in the reference layout: child[8*num_nodes] (host), cells numbered
 * from n in pre-order, root children in child[0..7], leaves = original
 * particle indices; level[num_nodes] (host, optional); node COMs into the
 * host arrays x,y,z,m (num_nodes each, optional).  Returns the cell count in
 * *cells. */
int mhpc_export_tree(mhpc_ctx* ctx, int num_nodes, int* child, int* level, double* x, double* y,
                     double* z, double* m, int* cells);

/* Statistics of the last RHS (synchronises the stream). */
typedef struct mhpc_stats {
    int n;
    int cells;                 /* tree cells */
    int max_level;
    int key_collisions;        /* particles sharing a full 63-bit key with another */
    double bbox[6];
    double radius;
    double gravity_interactions; /* accepted particle-node interactions (walk) */
    double gravity_nodes_visited;
    double gravity_quad_interactions; /* accepted cells evaluated with a quadrupole term (mixed walk) */
    int max_noi;               /* largest neighbour count */
    double mean_noi;
    int sml_sweeps;            /* variable-h sweeps run */
    int sml_out_of_band;       /* particles whose final count misses the band */
    int predictor_used;        /* particles whose learned h was accepted */
    int predictor_fallback;    /* particles that fell back to the plain iteration */
    float ms_stage[12];        /* bbox_keys, sort, tree, com, gravity, frnn (list walk), sml (variable-h
                                  iteration), density, forces, band (band repair), unused, total */
    int sml_band_before;       /* particles out of the band before the band repair (-1: no repair ran) */
    int sml_band_skipped;      /* band repair rounds skipped because their pair changes overflowed the
                                  event buffer (4 per particle) */
    /* Totals over the right-hand sides of mhpc_rhs / mhpc_integrate since the
     * context was created or mhpc_stats_reset_run was called (SPH
     * configurations; the per-stage exports are not counted).  They are
     * accumulated on the device, so a caller reads them once after a run
     * instead of synchronising after every step. */
    int run_rhs;                       /* right-hand sides counted */
    int run_out_of_band_max;           /* largest sml_out_of_band of one RHS */
    double run_out_of_band_sum;        /* sum of sml_out_of_band */
    double run_band_before_sum;        /* sum of sml_band_before over the RHS that ran the repair */
    int run_band_rhs;                  /* RHS that ran the band repair */
    int run_pad;
    double run_predictor_used_sum;     /* sum of predictor_used */
    double run_predictor_fallback_sum; /* sum of predictor_fallback */
} mhpc_stats;
int mhpc_get_stats(mhpc_ctx* ctx, mhpc_stats* out);
/* Restart the run totals (run_* fields of mhpc_stats); stream-ordered. */
int mhpc_stats_reset_run(mhpc_ctx* ctx);

/* FP64 diagnostics (src/miluphpc.cpp:577-677, Physics::Kernel
 * src/subdomain_key_tree/subdomain.cu:2423-2644): out[0] kinetic energy,
 * out[1] internal energy sum m e, out[2..4] linear momentum, out[5..7]
 * angular momentum, out[8..10] centre of mass.  Synchronises. */
int mhpc_diagnostics(mhpc_ctx* ctx, const mhpc_particles* p, double* out11);

/* Gravitational potential phi_i (caller's order, into pot_dev when not NULL)
 * and potential energy W = 1/2 sum m_i phi_i (into *energy_out when not NULL)
 * of the particles' current positions: a tree build and the interaction-list
 * walk with the geometric rule (theta_mixed) whatever the configured
 * precision and opening rule, so that successive calls are comparable (energy
 * drift).  The caller's accelerations are not touched.  Synchronises.  The
 * reference has no potential on its path; this serves the energy diagnostics
 * next to mhpc_diagnostics. */
int mhpc_potential(mhpc_ctx* ctx, const mhpc_particles* p, double* pot_dev, double* energy_out);

/* Miluphpc::removeParticles (src/miluphpc.cpp:3216-3348) with
 * ParticlesNS::Kernel::mark2remove (src/subdomain_key_tree/subdomain.cu:2161-2240):
 * removes the particles outside the region of config remove_particles_criterion
 * (0: sqrt(x^2+y^2+z^2) < d kept, 1: |x|, |y|, |z| < d kept; d =
 * remove_particles_dimension) from every non-null array of *p (all FP64 fields,
 * noi and material_id; nnl and level are per-RHS outputs and are left alone),
 * keeping the order of the survivors and zeroing the vacated tail; p->n is
 * lowered accordingly.  The reference's integrators call it at the start of
 * each step when removeParticles is set; so should the caller of
 * mhpc_integrate.  Unlike the reference, the gravitational and leapfrog-old
 * accelerations and the rates are compacted too, so they stay with their
 * particles.  Synchronises the context's stream once. */
int mhpc_remove_particles(mhpc_ctx* ctx, mhpc_particles* p, int* n_removed);

/* FP64 direct summation for verification: accelerations of `nt` target
 * particles (original indices, device) from all n particles with softening
 * eps2; outputs are device arrays of nt doubles. */
int mhpc_direct_gravity(const double* x, const double* y, const double* z, const double* m, int n,
                        const int* targets, int nt, double eps2, double* gax, double* gay,
                        double* gaz, void* stream);
/* The same with a per-target softening added: target t uses eps2 +
 * eps2_targets[t] (device, nt doubles), e.g. (softening_h_factor h_i)^2 to
 * check the walks' h-tied softening rule. */
int mhpc_direct_gravity_soft(const double* x, const double* y, const double* z, const double* m, int n,
                             const int* targets, int nt, double eps2, const double* eps2_targets, double* gax,
                             double* gay, double* gaz, void* stream);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (independent
 * chains of the paired FFMA2 instruction, the form the mixed walk issues, on
 * every SM; the roofline denominator of the FP32 walk).
 * Allocates and frees a small buffer; synchronises. */
int mhpc_fp32_peak(double* tflops);

/* ------------------------------------------------ learned smoothing length */
/* MLP 12 -> 64 -> 64 -> 1 (SiLU), BF16 weights, FP32 accumulation, trained
 * on the GPU by the library's own tensor-core kernels; it predicts
 * log(h_next / h) from 12 per-particle features of the previous RHS.  Needs a
 * context created with cfg->learned_h (and variable_sml).  While it is
 * untrained every RHS runs the plain iteration and adds (features, converged
 * h) pairs to a training buffer; once trained, each RHS starts the iteration
 * from the predicted h and falls back to the plain iteration for particles
 * whose prediction misses the band.  Not in the reference. */
int mhpc_mlp_reset(mhpc_ctx* ctx, uint64_t seed);
/* `iters` Adam steps (mini-batches of 8192 pairs drawn from the training
 * buffer; features and target standardised with the buffer's statistics on
 * the first call); *loss_out (optional) receives the last mini-batch loss.
 * Returns MHPC_ERR_ARG while fewer than 1024 pairs are available.
 * Synchronises. */
int mhpc_mlp_train(mhpc_ctx* ctx, int iters, float lr, float* loss_out);
/* Parameter count; layout: W1[64][16] (inputs 12..15 zero), b1[64],
 * W2[64][64] (out, in), b2[64], w3[64], b3[1]. */
int mhpc_mlp_num_params(void);
/* Forward pass on `rows` raw feature rows (device, rows x 12 float) into out
 * (device, rows float, optional), and the FP32 gradient of the mean-squared
 * loss against target (device, rows float) w.r.t. all parameters into grad
 * (device, mhpc_mlp_num_params() floats, optional); *loss_out (host,
 * optional).  Synchronises. */
int mhpc_mlp_forward_backward(mhpc_ctx* ctx, const float* feats, int rows, const float* target,
                              float* out, float* grad, float* loss_out);
/* Copy the FP32 master weights out (host, mhpc_mlp_num_params() floats) or in. */
int mhpc_mlp_get_params(mhpc_ctx* ctx, float* host_params);
int mhpc_mlp_set_params(mhpc_ctx* ctx, const float* host_params);

#ifdef __cplusplus
}
#endif
#endif /* MHPC_H */
