// Context, orchestration and the C ABI of libmhpc.
//
// mhpc_rhs follows the single-rank sequence of Miluphpc::rhs()
// (src/miluphpc.cpp:387-562): bounding box, keys, sort, tree, centres of mass,
// gravity, SPH.  Differences by design: the work is stream-ordered with no
// device synchronisation between stages (the reference synchronises after
// every kernel, include/cuda_utils/cuda_launcher.cuh:114-141), the MPI
// domain-list / LET kernels that do no work on one rank are not run, and all
// workspace is allocated once in mhpc_ctx_create.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "gravity.cuh"
#include "integrate.cuh"
#include "mlp.cuh"
#include "sph.cuh"
#include "tree.cuh"

enum Stage { EV_START, EV_KEYS, EV_SORT, EV_TREE, EV_COM, EV_GRAV, EV_SML, EV_LISTS, EV_FRNN, EV_DENS, EV_FORCES, EV_END,
             EV_COUNT };

struct mhpc_ctx {
    int cap = 0, cell_cap = 0, cap_nodes = 0, maxnb = 180;
    int device = 0;
    mhpc_config cfg;
    mhpc_material mats[MHPC_MAX_MATERIALS];
    int nmat = 1;
    cudaStream_t stream = nullptr;
    DevStatus* st = nullptr;
    DevStatus* h_st = nullptr;
    long long* ord = nullptr;
    double* bbox = nullptr;
    uint64_t* keys = nullptr;
    uint64_t* skey = nullptr;
    int* perm = nullptr;
    void* sort_scratch = nullptr;
    size_t sort_bytes = 0;
    void* scan_scratch = nullptr;
    double *sx = nullptr, *sy = nullptr, *sz = nullptr, *sm = nullptr, *sh = nullptr;
    double *svx = nullptr, *svy = nullptr, *svz = nullptr, *se = nullptr, *srho = nullptr, *sp = nullptr,
           *scs = nullptr, *sbal = nullptr;
    float4 *sf0 = nullptr, *sf1 = nullptr, *sf2 = nullptr;  // FP32 pair-sum views (mixed SPH)
    float2* sf3 = nullptr;
    int* smat = nullptr;
    TreeDev T;
    int* nbr = nullptr;
    int* noi = nullptr;
    double* hold = nullptr;
    int *vh_done = nullptr, *vh_nit = nullptr, *vh_count = nullptr;
    int *vh_flags = nullptr, *vh_off = nullptr, *vh_list = nullptr;
    int *vh_list2 = nullptr, *vh_cnt = nullptr;  // alternating sweep lists and their lengths
    double* h_start = nullptr;  // sorted h the variable-h iteration started from
    double last_dt = 0.0;
    double* diag_part = nullptr;
    double* diag_out = nullptr;
    cudaEvent_t ev[EV_COUNT];
    bool ev_recorded[EV_COUNT];
    bool first_rhs_done = false;
    // stage bookkeeping for the per-stage exports: particle count of the last
    // tree build and of the last neighbour lists, multipoles present, the last
    // neighbour search started from the learned prediction
    int tree_n = -1, lists_n = -1;
    bool com_ready = false, quad_ready = false, frnn_learned = false;
    // neighbour-band repair: pair-change events, their counters, and whether
    // the last neighbour search ran the repair
    int2* band_ev = nullptr;
    int band_cap = 0;
    int* band_ctr = nullptr;
    double* band_h0 = nullptr;
    int* nb_appended = nullptr;  // [n] lists with appended entries (zero between calls)
    bool band_ran = false;
    bool dens_ready = false;  // the sorted rho, p, c_s are the density pass's of this tree
    // run totals of the per-RHS counters (SPH configurations); st_pending: *st
    // holds a finished RHS whose counters are not yet in *run
    RunTotals* run = nullptr;
    bool st_pending = false;
    // a right-hand side ran since the host last read *st
    bool status_unread = false;
    long long learned_rhs = 0;  // right-hand sides that ran the learned feature pass
    // particle count of the last gravity walk, -1 before the first: the
    // relative opening rule reads that walk's accelerations from g_ax/g_ay/g_az
    int grav_prev_n = -1;
    int last_n = 0;
    // predictor-corrector: predicted state (IntegratedParticles), step size on the device
    mhpc_particles pred;
    double* dt_dev = nullptr;
    double* dt_part = nullptr;
    double time = 0.0;
    // device mirrors for mhpc_integrate_host, used by alternate steps so that
    // one step's copy-in can run while the previous step computes
    mhpc_particles mirror[2];
    bool mirror_ready = false;
    // mhpc_potential: the tree gets walk records whatever the precision; scratch
    // for the potential and the walk's accelerations (allocated on first use)
    bool force_wrec = false;
    double* pot_scratch = nullptr;
    // mhpc_integrate_host, leapfrog: the drifted positions are copied out on
    // copy_stream while the right-hand side runs (pos_out = host x, y, z)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_drift = nullptr;
    // host-state steps: copy-in / copy-out streams and their events (per
    // mirror: compute done, and per field: copy-out done)
    cudaStream_t in_stream = nullptr, out_stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_computed[2] = {};
    cudaEvent_t ev_out[2][18 * 4] = {};  // [mirror][field * kHostChunks + chunk]
    bool out_pending[2][18 * 4] = {};
    bool computed_pending[2] = {};
    long long host_steps = 0;
    double* pos_out[3] = {nullptr, nullptr, nullptr};
    std::vector<void*> allocs;
    MlpState* mlp = nullptr;
};

namespace {

template <typename T>
int dalloc(mhpc_ctx* c, T** p, size_t count) {
    if (count == 0) count = 1;
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * count) != cudaSuccess) return MHPC_ERR_CUDA;
    c->allocs.push_back(q);
    *p = (T*)q;
    return MHPC_OK;
}

#define TRY(x)                 \
    do {                       \
        int _r = (x);          \
        if (_r) return _r;     \
    } while (0)

MatDev to_dev(const mhpc_material& m, int si_units) {
    MatDev d;
    d.eos_type = m.eos_type;
    d.interactions = m.interactions;
    d.alpha = m.alpha;
    d.beta = m.beta;
    d.K = m.polytropic_K;
    d.gamma = m.polytropic_gamma;
    d.rho0 = m.rho_0;
    d.bulk = m.bulk_modulus;
    d.n_exp = m.n;
    d.shear = m.shear_modulus;
    // initializeSoundSpeed (src/sph/soundspeed.cu:4-36)
    d.cs_init = 0.0;
    if (m.eos_type == 1 && m.rho_0 > 0) d.cs_init = std::sqrt(m.bulk_modulus / m.rho_0);
    if (m.eos_type == 3) d.cs_init = si_units ? 203.0 : 203.0 / 2.998e8;
    return d;
}

SphParams sph_params(const mhpc_ctx* c, int n) {
    SphParams P;
    std::memset(&P, 0, sizeof(P));
    P.n = n;
    P.maxnb = c->maxnb;
    P.kernel = c->cfg.smoothing_kernel;
    P.avg_h = (c->cfg.variable_sml || c->cfg.integrate_sml) ? 1 : 0;
    P.integrate_energy = c->cfg.integrate_energy;
    P.integrate_sml = c->cfg.integrate_sml;
    P.integrate_density = c->cfg.integrate_density;
    P.num_materials = c->nmat;
    P.mixed = c->cfg.precision >= 1;
    P.balsara = c->cfg.balsara ? 1 : 0;
    P.variable_sml = c->cfg.variable_sml ? 1 : 0;
    P.ord = c->ord;
    for (int i = 0; i < c->nmat && i < MHPC_MAX_MATERIALS; ++i) P.mat[i] = to_dev(c->mats[i], c->cfg.si_units);
    return P;
}

void record(mhpc_ctx* c, int e) {
    if (c->force_wrec) return;  // mhpc_potential's tree build: the last RHS keeps its stage times
    cudaEventRecord(c->ev[e], c->stream);
    c->ev_recorded[e] = true;
}

// softening_mode 1 with a positive factor: eps_i = softening_h_factor * h_i
bool h_softening(const mhpc_config& cfg) { return cfg.softening_mode == 1 && cfg.softening_h_factor > 0.0; }

int check_particles(const mhpc_ctx* c, const mhpc_particles* p) {
    if (!p) return MHPC_ERR_ARG;
    if (p->n < 0) return MHPC_ERR_ARG;
    if (p->n > c->cap) return MHPC_ERR_CAPACITY;
    if (p->n == 0) return MHPC_OK;
    if (!p->x || !p->y || !p->z || !p->mass) return MHPC_ERR_ARG;
    if (c->cfg.gravity && (!p->g_ax || !p->g_ay || !p->g_az)) return MHPC_ERR_ARG;
    // h-tied softening reads every particle's smoothing length
    if (c->cfg.gravity && h_softening(c->cfg) && !p->sml) return MHPC_ERR_ARG;
    if (c->cfg.sph && (!p->sml || !p->rho || !p->p || !p->cs || !p->ax || !p->ay || !p->az || !p->vx || !p->vy ||
                       !p->vz || !p->e))
        return MHPC_ERR_ARG;
    return MHPC_OK;
}

// bounding box, keys, sort, gather into SFC order, tree build
int stage_tree_build(mhpc_ctx* c, const mhpc_particles* p) {
    const int n = p->n;
    cudaStream_t s = c->stream;
    TRY(launch_bbox(p->x, p->y, p->z, n, c->ord, c->st, s));
    TRY(launch_bbox_finish(c->ord, c->bbox, s));
    TRY(launch_keys(p->x, p->y, p->z, n, c->ord, c->cfg.sfc, c->keys, nullptr, s));
    record(c, EV_KEYS);
    TRY(sort_pairs_u64(c->keys, nullptr, c->skey, c->perm, n, c->sort_scratch, c->sort_bytes, c->st, s));
    record(c, EV_SORT);
    GatherList L;
    std::memset(&L, 0, sizeof(L));
    const double* src[] = {p->x, p->y, p->z, p->mass};
    double* dst[] = {c->sx, c->sy, c->sz, c->sm};
    for (int a = 0; a < 4; ++a) { L.src[a] = src[a]; L.dst[a] = dst[a]; }
    L.count = 4;
    if (c->cfg.sph || (c->cfg.gravity && h_softening(c->cfg))) {
        L.src[L.count] = p->sml; L.dst[L.count++] = c->sh;
    }
    if (c->cfg.sph) {
        const double* s2[] = {p->vx, p->vy, p->vz};
        double* d2[] = {c->svx, c->svy, c->svz};
        for (int a = 0; a < 3; ++a) { L.src[L.count] = s2[a]; L.dst[L.count++] = d2[a]; }
        // e, rho, p and c_s are inputs of the density/EOS pass only where it
        // reads them: e and p for the ideal gas (p = (gamma - 1) rho e, its c_s
        // uses the previous p), rho when integrated, c_s for an EOS that does not
        // set it; else they are outputs or unused
        bool need_p = false, need_cs = false, need_e = false;
        for (int m = 0; m < c->nmat; ++m) {
            const int t = c->mats[m].eos_type;
            const bool known = t == 0 || t == 1 || t == 3 || t == 9 || t == 12;
            need_e = need_e || t == 9 || !known;
            need_p = need_p || t == 9 || !known;
            need_cs = need_cs || !known;
        }
        if (need_e) { L.src[L.count] = p->e; L.dst[L.count++] = c->se; }
        if (c->cfg.integrate_density) { L.src[L.count] = p->rho; L.dst[L.count++] = c->srho; }
        if (need_p) { L.src[L.count] = p->p; L.dst[L.count++] = c->sp; }
        if (need_cs) { L.src[L.count] = p->cs; L.dst[L.count++] = c->scs; }
        if (p->material_id) {
            // ids index the material table: out-of-range ids are an argument error
            L.isrc = p->material_id; L.idst = c->smat; L.imax = c->nmat; L.st = c->st;
        }
    }
    TRY(launch_gather(n, c->perm, L, s));
    c->T.n = n;
    TRY(tree_build(c->T, c->skey, c->scan_scratch, c->st, s));
    record(c, EV_TREE);
    c->tree_n = n;
    c->com_ready = c->quad_ready = false;
    c->dens_ready = false;
    return MHPC_OK;
}

// TreeNS::Kernel::calculateCentersOfMass (src/subdomain_key_tree/tree.cu:1416-1497)
// for all levels, plus the mixed walks' multipoles and walk records and the
// SPH node boxes, on the tree of the last stage_tree_build
int stage_com(mhpc_ctx* c) {
    const int want_quad = c->cfg.gravity && (c->cfg.precision >= 1 || c->force_wrec);
    TRY(tree_upward(c->T, c->sx, c->sy, c->sz, c->sm, want_quad, c->cfg.sph ? 1 : 0, c->ord, c->cfg.theta_mixed,
                    c->st, c->stream));
    record(c, EV_COM);
    c->com_ready = true;
    c->quad_ready = want_quad;
    return MHPC_OK;
}

int stage_tree(mhpc_ctx* c, const mhpc_particles* p) {
    TRY(stage_tree_build(c, p));
    return stage_com(c);
}

// precision: -1 the configured one, otherwise 0 plain FP64, 1 interaction
// lists, 2 per-lane vote (the mixed walks need the multipoles of stage_com)
int stage_gravity(mhpc_ctx* c, const mhpc_particles* p, int precision = -1) {
    if (precision < 0) precision = c->cfg.precision;
    if (precision > 2) return MHPC_ERR_ARG;
    if (precision >= 1 && !c->quad_ready) return MHPC_ERR_ARG;
    GravParams G;
    std::memset(&G, 0, sizeof(G));
    G.n = p->n;
    G.eps2 = c->cfg.smoothing;
    G.h_factor = h_softening(c->cfg) ? c->cfg.softening_h_factor : 0.0;
    G.G = c->cfg.si_units ? 6.67430e-11 : 1.0;
    G.ord = c->ord;
    if (precision == 1) {
        G.theta = c->cfg.theta_mixed;
        G.rel_alpha = (c->cfg.gravity_mac == 1 && c->grav_prev_n == p->n) ? c->cfg.mac_alpha : 0.0;
        G.quad_alpha = G.rel_alpha > 0.0 ? c->cfg.mac_quad_alpha : 0.0;
        TRY(gravity_lists(c->T, G, c->sx, c->sy, c->sz, c->sh, c->perm, p->g_ax, p->g_ay, p->g_az, c->st,
                          c->stream));
    } else if (precision == 2) {
        G.theta = c->cfg.theta_mixed;
        TRY(gravity_mixed(c->T, G, c->sx, c->sy, c->sz, c->sh, c->perm, p->g_ax, p->g_ay, p->g_az, c->st,
                          c->stream));
    } else if (c->cfg.gravity_force_version == 2) {
        G.theta = c->cfg.theta;
        TRY(gravity_v1(c->T, G, c->sh, c->perm, p->g_ax, p->g_ay, p->g_az, c->st, c->stream));
    } else {
        G.theta = c->cfg.theta;
        TRY(gravity_v2(c->T, G, c->sx, c->sy, c->sz, c->sh, c->perm, p->g_ax, p->g_ay, p->g_az, c->st,
                       c->stream));
    }
    c->grav_prev_n = p->n;
    record(c, EV_GRAV);
    return MHPC_OK;
}

int sph_target(const mhpc_ctx* c) { return c->mats[0].interactions > 0 ? c->mats[0].interactions : 50; }

SphSorted sph_sorted(mhpc_ctx* c, const mhpc_particles* p) {
    SphSorted S;
    S.x = c->sx; S.y = c->sy; S.z = c->sz; S.m = c->sm; S.h = c->sh;
    S.vx = c->svx; S.vy = c->svy; S.vz = c->svz; S.e = c->se;
    S.mat = p->material_id ? c->smat : nullptr;
    S.rho = c->srho; S.p = c->sp; S.cs = c->scs; S.bal = c->sbal;
    S.f0 = c->sf0; S.f1 = c->sf1; S.f2 = c->sf2; S.f3 = c->sf3;
    return S;
}

// SPH::fixedRadiusNN_variableSML (src/sph/sph.cu:739-961, Jacobi form) when
// variable_h, starting from the learned prediction when `predictor`, then
// SPH::fixedRadiusNN (src/sph/sph.cu:93-281): the neighbour lists
// The variable-h iteration runs on neighbour lists (sph_variable_h_lists; 0:
// count walks, then one list walk with the final h).
#ifndef MHPC_VH_LISTS
#define MHPC_VH_LISTS 1
#endif
int stage_frnn(mhpc_ctx* c, const mhpc_particles* p, bool variable_h, bool learned) {
    const int n = p->n;
    cudaStream_t s = c->stream;
    SphParams P = sph_params(c, n);
    const int target = sph_target(c);
    c->frnn_learned = learned && variable_h;
    if (variable_h) {
        CUDA_TRY(cudaMemsetAsync(c->vh_done, 0, sizeof(int) * n, s));
        CUDA_TRY(cudaMemsetAsync(c->vh_nit, 0xff, sizeof(int) * n, s));  // nit starts at -1
        CUDA_TRY(cudaMemcpyAsync(c->h_start, c->sh, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        // learned path: start the iteration from the predicted h; particles whose
        // prediction lands in the band stop after the first sweep
        if (learned) TRY(mlp_apply_prediction(c->mlp, c->perm, c->sh, n, s));
        VhBuffers B;
        B.hold = c->hold; B.done = c->vh_done; B.nit = c->vh_nit; B.count = c->vh_count;
        B.flags = c->vh_flags; B.off = c->vh_off; B.list = c->vh_list; B.scan_scratch = c->scan_scratch;
        B.list2 = c->vh_list2; B.cnt = c->vh_cnt;
        if (MHPC_VH_LISTS) {
            // the iteration on lists: its lists are the right-hand side's
            BandBuffers E;
            std::memset(&E, 0, sizeof(E));
            E.dirty = c->vh_count; E.hnew = c->hold; E.events = c->band_ev; E.cap_events = c->band_cap;
            E.ctr = c->band_ctr; E.scan_scratch = c->scan_scratch; E.appended = c->nb_appended;
            TRY(sph_variable_h_lists(c->T, P, c->sx, c->sy, c->sz, c->sh, c->nbr, c->noi, B, E, target,
                                     c->cfg.nb_tolerance, c->cfg.max_sml_iterations,
                                     c->cfg.max_sml_iterations + 2, c->st, s));
        } else {
            TRY(sph_variable_h(c->T, P, c->sx, c->sy, c->sz, c->sh, B, target, c->cfg.nb_tolerance,
                               c->cfg.max_sml_iterations, c->cfg.max_sml_iterations + 2, c->st, s));
        }
        GatherList L;
        std::memset(&L, 0, sizeof(L));
        L.count = 1;
        L.src[0] = c->sh;
        L.dst[0] = p->sml;
        TRY(launch_scatter(n, c->perm, L, s));
        if (learned)
            TRY(mlp_collect(c->mlp, c->perm, c->h_start, c->sh, MHPC_VH_LISTS ? c->noi : c->vh_count, c->vh_nit,
                            target, c->cfg.nb_tolerance, c->cfg.max_sml_iterations, n, s));
    }
    record(c, EV_SML);
    SphSorted S = sph_sorted(c, p);
    if (!(variable_h && MHPC_VH_LISTS)) TRY(sph_frnn(c->T, P, S, c->nbr, c->noi, c->st, s));
    record(c, EV_LISTS);
    c->band_ran = false;
    if (variable_h && c->cfg.sml_band_rounds > 0) {
        // counts that drifted out of the band: repaired on the lists, then the
        // final h goes back to the caller's order
        BandBuffers B;
        B.flags = c->vh_flags; B.off = c->vh_off; B.list = c->vh_list; B.dirty = c->vh_done; B.hnew = c->hold;
        B.events = c->band_ev; B.cap_events = c->band_cap; B.ctr = c->band_ctr; B.scan_scratch = c->scan_scratch;
        B.h0 = c->band_h0;
        B.appended = c->nb_appended;
        TRY(sph_band_fixup(c->T, P, c->sx, c->sy, c->sz, c->sh, c->nbr, c->noi, B, target, c->cfg.nb_tolerance,
                           c->cfg.sml_band_rounds, c->st, s));
        GatherList L;
        std::memset(&L, 0, sizeof(L));
        L.count = 1;
        L.src[0] = c->sh;
        L.dst[0] = p->sml;
        TRY(launch_scatter(n, c->perm, L, s));
        c->band_ran = true;
    }
    record(c, EV_FRNN);
    c->lists_n = n;
    return MHPC_OK;
}

// SPH::Kernel::calculateDensity (src/sph/density.cu:8-72), calculateSoundSpeed
// (src/sph/soundspeed.cu:38-97) and calculatePressure (src/sph/pressure.cu:5-87)
// over the lists of stage_frnn, plus the Balsara factors when configured
int stage_density_eos(mhpc_ctx* c, const mhpc_particles* p) {
    SphParams P = sph_params(c, p->n);
    SphSorted S = sph_sorted(c, p);
    TRY(sph_density_eos(P, S, c->nbr, c->noi, c->perm, p->rho, p->p, p->cs, c->st, c->stream));
    if (c->cfg.balsara) TRY(sph_balsara(P, S, c->nbr, c->noi, c->st, c->stream));
    record(c, EV_DENS);
    c->dens_ready = true;
    return MHPC_OK;
}

// SPH::Kernel::internalForces (src/sph/internal_forces.cu:4-668) over the
// lists of stage_frnn; the reference-layout lists and counts when the SoA
// asks for them; the band statistic after a variable-h search; the learned
// predictor's features and its prediction for the next right-hand side
int stage_forces(mhpc_ctx* c, const mhpc_particles* p) {
    const int n = p->n;
    cudaStream_t s = c->stream;
    SphParams P = sph_params(c, n);
    SphSorted S = sph_sorted(c, p);
    const int target = sph_target(c);
    const bool learned = c->frnn_learned;
    TRY(sph_forces(P, S, c->nbr, c->noi, c->perm, p->ax, p->ay, p->az, p->drhodt, p->dedt, p->dsmldt, c->st, s));
    if (p->nnl || p->noi) TRY(sph_export_nnl(P, c->nbr, c->noi, c->perm, p->nnl, p->noi, s));
    if (c->cfg.variable_sml) TRY(sph_band_stats(P, c->noi, target, c->cfg.nb_tolerance, c->st, s));
    record(c, EV_FORCES);
    if (learned) {
        MlpFeatureInputs in;
        in.n = n; in.perm = c->perm; in.h = c->sh; in.h_start = c->h_start; in.rho = c->srho; in.cs = c->scs;
        in.vx = c->svx; in.vy = c->svy; in.vz = c->svz; in.noi = c->noi; in.nit = c->vh_nit;
        in.ax = p->ax; in.ay = p->ay; in.az = p->az;
        in.gx = c->cfg.gravity ? p->g_ax : nullptr; in.gy = p->g_ay; in.gz = p->g_az;
        in.drhodt = p->drhodt; in.m = c->sm;
        in.dt = c->last_dt > 0 ? c->last_dt : (c->cfg.time_step > 0 ? c->cfg.time_step : 1.0);
        in.target = target;
        // the predictor follows the flow: a few Adam steps on the recent pairs
        // every learned_refresh_every right-hand sides (queued, no sync)
        ++c->learned_rhs;
        if (c->cfg.learned_refresh_every > 0 && c->learned_rhs % c->cfg.learned_refresh_every == 0)
            TRY(mlp_refresh(c->mlp, c->cfg.learned_refresh_iters, 1e-3f, 8192, s));
        TRY(mlp_features_predict(c->mlp, in, s));
    }
    return MHPC_OK;
}

int stage_sph(mhpc_ctx* c, const mhpc_particles* p) {
    TRY(stage_frnn(c, p, c->cfg.variable_sml != 0, c->cfg.learned_h && c->mlp));
    TRY(stage_density_eos(c, p));
    return stage_forces(c, p);
}

// Zero the status word on the stream; with SPH the counters of a finished
// right-hand side are first added to the run totals (one small kernel).
// Start of a right-hand side.  A status the host has not read since the
// previous right-hand side (queued host-state steps, the predictor-corrector's
// second RHS) keeps its error code, so no error is lost between reads.
int reset_status(mhpc_ctx* c, cudaStream_t s) {
    const int keep = c->status_unread ? 1 : 0;
    if (c->cfg.sph || keep) {
        TRY(launch_status_fold(c->st, c->run, c->st_pending ? 1 : 0, c->band_ran ? 1 : 0, keep, s));
    } else {
        CUDA_TRY(cudaMemsetAsync(c->st, 0, sizeof(DevStatus), s));
    }
    c->st_pending = false;
    return MHPC_OK;
}

int rhs_async(mhpc_ctx* c, const mhpc_particles* p, int self_gravity) {
    TRY(check_particles(c, p));
    for (int e = 0; e < EV_COUNT; ++e) c->ev_recorded[e] = false;
    c->last_n = p->n;
    if (p->n == 0) return MHPC_OK;
    TRY(reset_status(c, c->stream));
    record(c, EV_START);
    TRY(stage_tree(c, p));
    if (c->cfg.gravity && self_gravity) TRY(stage_gravity(c, p));
    if (c->cfg.sph) TRY(stage_sph(c, p));
    record(c, EV_END);
    c->first_rhs_done = true;
    c->st_pending = c->cfg.sph != 0;
    c->status_unread = true;
    return MHPC_OK;
}

int read_status(mhpc_ctx* c) {
    CUDA_TRY(cudaMemcpyAsync(c->h_st, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->status_unread = false;
    return c->h_st->code;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* mhpc_status_string(int s) {
    switch (s) {
        case MHPC_OK: return "ok";
        case MHPC_ERR_ARG: return "invalid argument";
        case MHPC_ERR_CUDA: return "CUDA runtime error";
        case MHPC_ERR_CAPACITY: return "particle count exceeds context capacity";
        case MHPC_ERR_NODE_POOL: return "tree node pool exhausted";
        case MHPC_ERR_DEPTH: return "traversal depth exceeded";
        case MHPC_ERR_NEIGHBOURS: return "too many neighbours (max_num_interactions)";
        case MHPC_ERR_NAN: return "non-finite position or non-positive density";
        case MHPC_ERR_CONFIG: return "configuration file missing or malformed";
        case MHPC_ERR_NO_DEVICE: return "no CUDA device";
        case MHPC_ERR_TIMEOUT: return "bounded device wait ran out";
        case MHPC_ERR_UNSUPPORTED: return "unsupported option";
        default: return "unknown status";
    }
}

int mhpc_version(void) { return 1; }

int mhpc_bbox(const double* x, const double* y, const double* z, int n, double* bbox_dev, void* stream) {
    if (n < 0 || !bbox_dev || (n > 0 && (!x || !y || !z))) return MHPC_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    // the ordered-integer (min, max) pair is reduced in the first 16 bytes of
    // the caller's 48-byte output and expanded in place
    long long* ord = reinterpret_cast<long long*>(bbox_dev);
    TRY(launch_bbox(x, y, z, n, ord, nullptr, s));
    TRY(launch_bbox_finish(ord, bbox_dev, s));
    return MHPC_OK;
}

int mhpc_keys(const double* x, const double* y, const double* z, int n, const double* bbox_dev, int curve,
              uint64_t* keys, void* stream) {
    if (n < 0 || !bbox_dev || !keys || curve < 0 || curve > 1 || (n > 0 && (!x || !y || !z))) return MHPC_ERR_ARG;
    return launch_keys_box(x, y, z, n, bbox_dev, curve, keys, (cudaStream_t)stream);
}

size_t mhpc_sort_scratch_bytes(int n) { return n < 0 ? 0 : sort_scratch_bytes(n) + 256; }

// The last 256 bytes of the scratch hold a status word: nonzero (MHPC_ERR_TIMEOUT)
// if a bounded look-back wait ran out.
int mhpc_sort_pairs(const uint64_t* keys_in, const int* vals_in, uint64_t* keys_out, int* vals_out, int n,
                    void* scratch, size_t scratch_bytes, void* stream) {
    if (n < 0 || !scratch) return MHPC_ERR_ARG;
    if (scratch_bytes < mhpc_sort_scratch_bytes(n)) return MHPC_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    DevStatus* st = reinterpret_cast<DevStatus*>((char*)scratch + sort_scratch_bytes(n));
    CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(DevStatus), s));
    return sort_pairs_u64(keys_in, vals_in, keys_out, vals_out, n, scratch, sort_scratch_bytes(n), st, s);
}

int mhpc_ctx_create(mhpc_ctx** out, int capacity, const mhpc_config* cfg, const mhpc_material* materials,
                    int num_materials) {
    if (!out || capacity <= 0 || !cfg || num_materials < 0 || num_materials > MHPC_MAX_MATERIALS)
        return MHPC_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MHPC_ERR_NO_DEVICE;
    mhpc_ctx* c = new mhpc_ctx();
    c->cfg = *cfg;
    cudaGetDevice(&c->device);
    c->cap = capacity;
    c->maxnb = cfg->max_num_interactions > 0 ? cfg->max_num_interactions : 180;
    double f = cfg->node_pool_factor > 0 ? cfg->node_pool_factor : 1.0;
    c->cell_cap = (int)std::min(2147483000.0 - capacity, f * capacity + 20000.0);
    c->cap_nodes = capacity + c->cell_cap;
    if (num_materials == 0) {
        std::memset(c->mats, 0, sizeof(c->mats));
        c->mats[0].polytropic_gamma = 5.0 / 3.0;
        c->mats[0].eos_type = 9;
        c->mats[0].interactions = 60;
        c->nmat = 1;
    } else {
        for (int i = 0; i < num_materials; ++i) c->mats[i] = materials[i];
        c->nmat = num_materials;
    }
    int rc = MHPC_OK;
    const size_t n = capacity, M = c->cap_nodes;
#define A(p, cnt) \
    if (!rc) rc = dalloc(c, &(p), (cnt))
    A(c->st, 1);
    A(c->run, 1);
    A(c->ord, 2);
    A(c->bbox, 6);
    A(c->keys, n);
    A(c->skey, n);
    A(c->perm, n);
    c->sort_bytes = sort_scratch_bytes(capacity);
    {
        char* q = nullptr;
        A(q, c->sort_bytes);
        c->sort_scratch = q;
        char* r = nullptr;
        A(r, scan_scratch_bytes(capacity) + 256);
        c->scan_scratch = r;
    }
    A(c->sx, n); A(c->sy, n); A(c->sz, n); A(c->sm, n); A(c->sh, n);
    TreeDev& T = c->T;
    T.n = 0;
    T.cap_nodes = c->cap_nodes;
    A(T.dl, n); A(T.cnt, n); A(T.off, n + 1); A(T.leaf_node, n);
    A(T.link, M); A(T.first, M); A(T.last, M); A(T.parent, M);
    A(T.kids, 8 * M); A(T.kmask, M);
    A(T.com, M); A(T.bmin, M); A(T.bmax, M); A(T.hmax, M); A(T.arrive, M);
    A(T.nodes, 1);
    if (cfg->gravity) {
        A(T.wrec, 4 * M);
    }
    if (cfg->sph) {
        A(c->svx, n); A(c->svy, n); A(c->svz, n); A(c->se, n); A(c->srho, n); A(c->sp, n); A(c->scs, n);
        A(c->sbal, n);
        A(c->sf0, n); A(c->sf1, n); A(c->sf2, n); A(c->sf3, n);
        A(c->smat, n);
        size_t groups = (n + 31) / 32;
        A(c->nbr, groups * 32 * (size_t)c->maxnb);
        A(c->noi, n);
        A(c->hold, n); A(c->vh_done, n); A(c->vh_nit, n); A(c->vh_count, n);
        A(c->vh_flags, n); A(c->vh_off, n + 1); A(c->vh_list, n); A(c->h_start, n);
        A(c->vh_list2, n); A(c->vh_cnt, 2);
        // band repair events: a round changes a few pairs per out-of-band particle
        // (room for 4 per particle: a round that needs more is skipped and counted)
        c->band_cap = (int)std::min<size_t>(2147483000, std::max<size_t>(4096, 4 * n));
        A(c->band_ev, c->band_cap);
        A(c->band_ctr, 4);
        A(c->band_h0, n);
        A(c->nb_appended, n);
    }
    // mhpc_potential: the potential (when the caller passes no buffer) and the
    // walk's own accelerations, so that the caller's g_a stay untouched
    if (cfg->gravity) A(c->pot_scratch, 4 * n);
    A(c->diag_part, diagnostics_scratch_doubles());
    A(c->diag_out, 16);
    A(c->dt_dev, 1);
    A(c->dt_part, 148 * 2 * 6 + 16);
    std::memset(&c->pred, 0, sizeof(c->pred));
    if (cfg->integrator == 1) {
        mhpc_particles& q = c->pred;
        A(q.x, n); A(q.y, n); A(q.z, n); A(q.mass, n); A(q.vx, n); A(q.vy, n); A(q.vz, n);
        if (cfg->sph) {
            A(q.ax, n); A(q.ay, n); A(q.az, n); A(q.sml, n); A(q.rho, n); A(q.p, n); A(q.cs, n); A(q.e, n);
            A(q.drhodt, n); A(q.dedt, n); A(q.dsmldt, n);
        }
    }
#undef A
    if (!rc && cudaMallocHost(&c->h_st, sizeof(DevStatus)) != cudaSuccess) rc = MHPC_ERR_CUDA;
    for (int e = 0; e < EV_COUNT && !rc; ++e)
        if (cudaEventCreate(&c->ev[e]) != cudaSuccess) rc = MHPC_ERR_CUDA;
    if (!rc && cfg->learned_h) {
        rc = mlp_create(&c->mlp, capacity);
        if (!rc) rc = mlp_reset(c->mlp, 0x6d6c70ULL, c->stream);
    }
    if (rc) {
        mhpc_ctx_destroy(c);
        return rc;
    }
    CUDA_TRY(cudaMemset(c->st, 0, sizeof(DevStatus)));
    CUDA_TRY(cudaMemset(c->run, 0, sizeof(RunTotals)));
    if (c->nb_appended) CUDA_TRY(cudaMemset(c->nb_appended, 0, sizeof(int) * n));
    *out = c;
    return MHPC_OK;
}

int mhpc_ctx_destroy(mhpc_ctx* c) {
    if (!c) return MHPC_ERR_ARG;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaDeviceSynchronize();
    for (void* p : c->allocs) cudaFree(p);
    if (c->h_st) cudaFreeHost(c->h_st);
    for (int e = 0; e < EV_COUNT; ++e)
        if (c->ev[e]) cudaEventDestroy(c->ev[e]);
    if (c->mlp) mlp_destroy(c->mlp);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->ev_drift) cudaEventDestroy(c->ev_drift);
    for (cudaStream_t q : {c->in_stream, c->out_stream})
        if (q) {
            cudaStreamSynchronize(q);
            cudaStreamDestroy(q);
        }
    for (cudaEvent_t e : {c->ev_in, c->ev_computed[0], c->ev_computed[1]})
        if (e) cudaEventDestroy(e);
    for (auto& row : c->ev_out)
        for (cudaEvent_t e : row)
            if (e) cudaEventDestroy(e);
    if (c->mirror_ready) {
        for (mhpc_particles& m : c->mirror) {
            double** ptrs[] = {&m.x, &m.y, &m.z, &m.mass, &m.vx, &m.vy, &m.vz, &m.ax, &m.ay, &m.az, &m.g_ax,
                               &m.g_ay, &m.g_az, &m.g_ax_old, &m.g_ay_old, &m.g_az_old, &m.sml, &m.rho, &m.p,
                               &m.cs, &m.e, &m.drhodt, &m.dedt, &m.dsmldt};
            for (auto pp : ptrs)
                if (*pp) cudaFree(*pp);
        }
    }
    delete c;
    return MHPC_OK;
}

int mhpc_ctx_set_stream(mhpc_ctx* c, void* stream) {
    if (!c) return MHPC_ERR_ARG;
    c->stream = (cudaStream_t)stream;
    return MHPC_OK;
}

int mhpc_ctx_set_config(mhpc_ctx* c, const mhpc_config* cfg) {
    if (!c || !cfg) return MHPC_ERR_ARG;
    // max_num_interactions 0 means the default 180, as in mhpc_ctx_create
    const int maxnb = cfg->max_num_interactions > 0 ? cfg->max_num_interactions : 180;
    if ((cfg->sph && !c->cfg.sph) || (cfg->gravity && !c->cfg.gravity) ||
        (cfg->learned_h && !c->mlp) || maxnb != c->maxnb)
        return MHPC_ERR_ARG;  // would need buffers the context did not allocate
    c->cfg = *cfg;
    return MHPC_OK;
}

int mhpc_rhs_async(mhpc_ctx* c, const mhpc_particles* p, int step, int self_gravity) {
    (void)step;
    if (!c) return MHPC_ERR_ARG;
    return rhs_async(c, p, self_gravity);
}

int mhpc_ctx_status(mhpc_ctx* c) {
    if (!c) return MHPC_ERR_ARG;
    return read_status(c);
}

int mhpc_rhs(mhpc_ctx* c, const mhpc_particles* p, int step, int self_gravity, void* stream, float* ms_out) {
    if (!c) return MHPC_ERR_ARG;
    c->stream = (cudaStream_t)stream;
    TRY(mhpc_rhs_async(c, p, step, self_gravity));
    int code = read_status(c);
    if (ms_out) {
        *ms_out = 0.f;
        if (c->ev_recorded[EV_START] && c->ev_recorded[EV_END])
            cudaEventElapsedTime(ms_out, c->ev[EV_START], c->ev[EV_END]);
    }
    return code;
}

int mhpc_stage_tree(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    TRY(reset_status(c, c->stream));
    c->last_n = p->n;
    return stage_tree(c, p);
}

int mhpc_stage_gravity(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c || !c->cfg.gravity) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    return stage_gravity(c, p);
}

int mhpc_tree_build(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    TRY(reset_status(c, c->stream));
    for (int e = 0; e < EV_COUNT; ++e) c->ev_recorded[e] = false;
    c->last_n = p->n;
    record(c, EV_START);
    return stage_tree_build(c, p);
}

int mhpc_com(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    if (c->tree_n != p->n) return MHPC_ERR_ARG;  // mhpc_tree_build first
    return stage_com(c);
}

int mhpc_gravity(mhpc_ctx* c, const mhpc_particles* p, int precision) {
    if (!c || !c->cfg.gravity || precision < -1 || precision > 2) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    if (c->tree_n != p->n || !c->com_ready) return MHPC_ERR_ARG;  // mhpc_tree_build + mhpc_com first
    return stage_gravity(c, p, precision);
}

int mhpc_frnn(mhpc_ctx* c, const mhpc_particles* p, int variable_h, int predictor) {
    if (!c || !c->cfg.sph || (predictor && !c->mlp)) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    if (c->tree_n != p->n || !c->com_ready) return MHPC_ERR_ARG;
    return stage_frnn(c, p, variable_h != 0, predictor != 0);
}

int mhpc_density_eos(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c || !c->cfg.sph) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    if (c->lists_n != p->n) return MHPC_ERR_ARG;  // mhpc_frnn first
    return stage_density_eos(c, p);
}

int mhpc_forces(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c || !c->cfg.sph) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    if (c->lists_n != p->n) return MHPC_ERR_ARG;
    if (!c->dens_ready) {
        // forces on the caller's rho, p and c_s (mhpc_density_eos did not run
        // after this tree): their sorted copies, which the tree's gather leaves
        // out where the density pass would compute them
        GatherList L;
        std::memset(&L, 0, sizeof(L));
        const double* src[] = {p->rho, p->p, p->cs};
        double* dst[] = {c->srho, c->sp, c->scs};
        for (int a = 0; a < 3; ++a) { L.src[a] = src[a]; L.dst[a] = dst[a]; }
        L.count = 3;
        TRY(launch_gather(p->n, c->perm, L, c->stream));
    }
    TRY(stage_forces(c, p));
    record(c, EV_END);
    return MHPC_OK;
}

int mhpc_integrate_leapfrog(mhpc_ctx* c, const mhpc_particles* p, double dt, int half) {
    if (!c || !p || p->n < 0 || (half != 0 && half != 1)) return MHPC_ERR_ARG;
    if (p->n == 0) return MHPC_OK;
    if (!p->x || !p->y || !p->z || !p->vx || !p->vy || !p->vz || !p->g_ax || !p->g_ay || !p->g_az ||
        !p->g_ax_old || !p->g_ay_old || !p->g_az_old)
        return MHPC_ERR_ARG;
    return half == 0 ? launch_leapfrog_x(*p, dt, c->stream) : launch_leapfrog_v(*p, dt, c->stream);
}

int mhpc_integrate_euler(mhpc_ctx* c, const mhpc_particles* p, double dt) {
    if (!c || !p || p->n < 0) return MHPC_ERR_ARG;
    if (p->n == 0) return MHPC_OK;
    const mhpc_config& f = c->cfg;
    if (!p->x || !p->y || !p->z || !p->vx || !p->vy || !p->vz) return MHPC_ERR_ARG;
    if (f.gravity && (!p->g_ax || !p->g_ay || !p->g_az)) return MHPC_ERR_ARG;
    if (f.sph && (!p->ax || !p->ay || !p->az)) return MHPC_ERR_ARG;
    if (f.sph && ((f.integrate_density && (!p->rho || !p->drhodt)) || (f.integrate_energy && (!p->e || !p->dedt)) ||
                  (f.integrate_sml && (!p->sml || !p->dsmldt))))
        return MHPC_ERR_ARG;
    return launch_euler(*p, dt, f.gravity, f.sph, f.sph && f.integrate_density, f.sph && f.integrate_energy,
                        f.sph && f.integrate_sml, c->stream);
}

int mhpc_integrate_pc_step_size(mhpc_ctx* c, const mhpc_particles* p, double time_left, double* dt_dev) {
    if (!c || !p || !dt_dev || p->n <= 0) return MHPC_ERR_ARG;
    if (!p->sml || !p->vx || !p->vy || !p->vz) return MHPC_ERR_ARG;
    if (c->cfg.gravity && (!p->g_ax || !p->g_ay || !p->g_az)) return MHPC_ERR_ARG;
    if (c->cfg.sph && (!p->ax || !p->ay || !p->az || !p->cs || !p->rho || !p->drhodt)) return MHPC_ERR_ARG;
    if (c->cfg.max_time_step <= 0) return MHPC_ERR_CONFIG;
    return launch_set_time_step(*p, c->cfg.gravity, c->cfg.sph, c->mats[0].alpha, c->mats[0].beta,
                                c->cfg.integrate_density, time_left, c->cfg.max_time_step, c->dt_part, dt_dev,
                                c->stream);
}

int mhpc_integrate_pc_predictor(mhpc_ctx* c, const mhpc_particles* p, const mhpc_particles* q, const double* dt_dev) {
    if (!c || !p || !q || !dt_dev || p->n < 0 || q->n < p->n) return MHPC_ERR_ARG;
    if (p->n == 0) return MHPC_OK;
    if (!p->g_ax || !p->g_ay || !p->g_az || !q->x || !q->y || !q->z || !q->vx || !q->vy || !q->vz || !q->mass)
        return MHPC_ERR_ARG;
    if (c->cfg.sph && (!q->sml || !q->cs || !q->rho || !q->p || !q->e || !p->ax)) return MHPC_ERR_ARG;
    return launch_pc_predictor(*p, *q, dt_dev, c->cfg.sph, c->cfg.integrate_density, c->cfg.integrate_energy,
                               c->stream);
}

int mhpc_integrate_pc_corrector(mhpc_ctx* c, const mhpc_particles* p, const mhpc_particles* q, const double* dt_dev) {
    if (!c || !p || !q || !dt_dev || p->n < 0 || q->n < p->n) return MHPC_ERR_ARG;
    if (p->n == 0) return MHPC_OK;
    if (!p->g_ax || !p->g_ay || !p->g_az || !q->vx || !q->vy || !q->vz) return MHPC_ERR_ARG;
    if (c->cfg.sph && (!q->ax || !q->sml || !q->drhodt || !q->dedt || !q->dsmldt || !p->ax || !p->sml))
        return MHPC_ERR_ARG;
    return launch_pc_corrector(*p, *q, dt_dev, c->cfg.sph, c->cfg.integrate_density, c->cfg.integrate_energy,
                               c->cfg.integrate_sml, c->stream);
}

int mhpc_stage_sph(mhpc_ctx* c, const mhpc_particles* p) {
    if (!c || !c->cfg.sph) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (p->n == 0) return MHPC_OK;
    return stage_sph(c, p);
}

}  // extern "C"

namespace {
// One integrator step; with `sync` false (host-state steps) it returns after
// queueing the work, without reading the status word, except where the host
// needs a device value (the predictor-corrector's step size, the status after
// the leapfrog's initial right-hand side).
int integrate_step(mhpc_ctx* c, const mhpc_particles* p, int step, double* dt_out, bool sync);
}  // namespace

extern "C" {

int mhpc_integrate(mhpc_ctx* c, const mhpc_particles* p, int step, double* dt_out) {
    return integrate_step(c, p, step, dt_out, true);
}

}  // extern "C"

namespace {
int integrate_step(mhpc_ctx* c, const mhpc_particles* p, int step, double* dt_out, bool sync) {
    if (!c) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    const double dt = c->cfg.time_step;
    cudaStream_t s = c->stream;
    if (dt_out) *dt_out = dt;
    if (p->n == 0) return MHPC_OK;
    switch (c->cfg.integrator) {
        case 2: {  // Leapfrog::integrate (src/integrator/leapfrog.cpp:21-117)
            if (!p->g_ax_old || !p->g_ay_old || !p->g_az_old) return MHPC_ERR_ARG;
            if (step == 0 && !c->first_rhs_done) {
                TRY(rhs_async(c, p, 1));
                int code = read_status(c);
                if (code) return code;
            }
            TRY(launch_leapfrog_x(*p, dt, s));
            if (c->pos_out[0]) {
                // positions are final after the drift: copy them out while the
                // right-hand side (which only reads them) runs
                const size_t b = sizeof(double) * p->n;
                CUDA_TRY(cudaEventRecord(c->ev_drift, s));
                CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->ev_drift, 0));
                const double* src[3] = {p->x, p->y, p->z};
                for (int d = 0; d < 3; ++d)
                    CUDA_TRY(cudaMemcpyAsync(c->pos_out[d], src[d], b, cudaMemcpyDeviceToHost, c->copy_stream));
            }
            TRY(rhs_async(c, p, 1));
            TRY(launch_leapfrog_v(*p, dt, s));
        } break;
        case 0: {  // ExplicitEuler::integrate (src/integrator/explicit_euler.cpp:17-99)
            TRY(rhs_async(c, p, 1));
            TRY(launch_euler(*p, dt, c->cfg.gravity, c->cfg.sph, c->cfg.integrate_density, c->cfg.integrate_energy,
                             c->cfg.integrate_sml, s));
        } break;
        case 1: {  // PredictorCorrectorEuler::integrate (src/integrator/predictor_corrector_euler.cpp:47-151)
            if (!c->pred.x) return MHPC_ERR_ARG;  // context created for another integrator
            // the update kernels read g_a (zero without gravity, as in the reference) and the
            // step size reads every h
            if (!p->g_ax || !p->g_ay || !p->g_az || !p->sml) return MHPC_ERR_ARG;
            const int sph = c->cfg.sph;
            TRY(rhs_async(c, p, 1));
            const double alpha = c->mats[0].alpha, beta = c->mats[0].beta;
            const double time_left = c->cfg.time_end > c->time ? c->cfg.time_end - c->time : c->cfg.max_time_step;
            if (c->cfg.time_step > 0 && c->cfg.max_time_step <= 0) return MHPC_ERR_CONFIG;
            TRY(launch_set_time_step(*p, c->cfg.gravity, sph, alpha, beta, c->cfg.integrate_density, time_left,
                                     c->cfg.max_time_step, c->dt_part, c->dt_dev, s));
            mhpc_particles q = c->pred;
            q.n = p->n;
            q.num_nodes = p->n;
            // gravity is not recomputed on the predicted state (rhs(step, false, false));
            // the walk outputs are not read, the stored g_a is reused by the corrector
            q.g_ax = p->g_ax; q.g_ay = p->g_ay; q.g_az = p->g_az;
            q.noi = nullptr; q.nnl = nullptr; q.level = nullptr;
            q.material_id = p->material_id;
            TRY(launch_pc_predictor(*p, q, c->dt_dev, sph, c->cfg.integrate_density, c->cfg.integrate_energy, s));
            TRY(rhs_async(c, &q, 0));
            TRY(launch_pc_corrector(*p, q, c->dt_dev, sph, c->cfg.integrate_density, c->cfg.integrate_energy,
                                    c->cfg.integrate_sml, s));
            double h_dt = 0.0;
            CUDA_TRY(cudaMemcpyAsync(&h_dt, c->dt_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
            int code = read_status(c);
            if (dt_out) *dt_out = h_dt;
            c->time += h_dt;
            c->last_dt = h_dt;
            return code;
        }
        default:
            return MHPC_ERR_UNSUPPORTED;
    }
    c->time += dt;
    c->last_dt = dt;
    return sync ? read_status(c) : MHPC_OK;
}
}  // namespace

extern "C" {

// Host-state steps.  Successive steps use the two device mirrors in turn,
// and every field moves on its own schedule: a field goes in on `in_stream`
// once its mirror is free (the compute and the copy-out of the step before
// the previous one are done) and the host buffer holds the previous step's
// value (that step's copy-out of the field has landed; the host state is read
// and written in place); the outputs go out on `out_stream` after the
// compute, velocities first.  Steps are queued without waiting, so the next
// step's masses and (leapfrog) drifted positions go in while this step still
// computes, and its velocities and accelerations go in as soon as they are
// out (the bus is full duplex), piece by piece; the compute of a step starts
// when its inputs are in.
enum HostField { HF_X, HF_Y, HF_Z, HF_M, HF_VX, HF_VY, HF_VZ, HF_GX, HF_GY, HF_GZ, HF_H, HF_E, HF_RHO, HF_P,
                 HF_CS, HF_AX, HF_AY, HF_AZ, HF_COUNT };
// Each field moves in this many pieces, each with its own copy-out event, so
// that the next step's copy-in of a piece follows the copy-out of the same
// piece rather than of the whole field.
constexpr int kHostChunks = 4;
static_assert(HF_COUNT * kHostChunks <= 18 * 4, "host-step event arrays too small");

int host_streams(mhpc_ctx* c) {
    if (c->in_stream) return MHPC_OK;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->in_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_computed[k], cudaEventDisableTiming));
        for (int f = 0; f < HF_COUNT * kHostChunks; ++f)
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_out[k][f], cudaEventDisableTiming));
    }
    return MHPC_OK;
}

int mhpc_integrate_host_async(mhpc_ctx* c, mhpc_particles* h, int step, double* dt_out) {
    if (!c || !h) return MHPC_ERR_ARG;
    if (h->n > c->cap || h->n < 0) return MHPC_ERR_CAPACITY;
    const size_t n = c->cap;
    if (!c->mirror_ready) {
        for (mhpc_particles& m : c->mirror) {
            std::memset(&m, 0, sizeof(m));
            double** ptrs[] = {&m.x, &m.y, &m.z, &m.mass, &m.vx, &m.vy, &m.vz, &m.g_ax, &m.g_ay, &m.g_az,
                               &m.g_ax_old, &m.g_ay_old, &m.g_az_old};
            for (auto pp : ptrs) CUDA_TRY(cudaMalloc(pp, sizeof(double) * n));
            if (c->cfg.sph) {
                double** p2[] = {&m.ax, &m.ay, &m.az, &m.sml, &m.rho, &m.p, &m.cs, &m.e, &m.drhodt, &m.dedt,
                                 &m.dsmldt};
                for (auto pp : p2) CUDA_TRY(cudaMalloc(pp, sizeof(double) * n));
            }
        }
        c->mirror_ready = true;
    }
    TRY(host_streams(c));
    const int k = (int)(c->host_steps & 1), j = 1 - k;  // this step's mirror, the previous step's
    mhpc_particles& m = c->mirror[k];
    m.n = h->n;
    m.num_nodes = h->n;
    cudaStream_t s = c->stream;
    auto piece = [&](int i) { return (size_t)h->n * i / kHostChunks; };  // first element of piece i
    struct Field { int id; double* d; double* hh; };
    // state in (positions, velocities, masses; leapfrog carries g_a between
    // steps), the fields whose host copy is ready earliest first
    std::vector<Field> in = {{HF_M, m.mass, h->mass}, {HF_X, m.x, h->x}, {HF_Y, m.y, h->y}, {HF_Z, m.z, h->z},
                             {HF_VX, m.vx, h->vx}, {HF_VY, m.vy, h->vy}, {HF_VZ, m.vz, h->vz}};
    if (c->cfg.integrator == 2) {
        in.push_back({HF_GX, m.g_ax, h->g_ax}); in.push_back({HF_GY, m.g_ay, h->g_ay});
        in.push_back({HF_GZ, m.g_az, h->g_az});
    }
    if (c->cfg.sph) {
        in.push_back({HF_H, m.sml, h->sml}); in.push_back({HF_E, m.e, h->e}); in.push_back({HF_RHO, m.rho, h->rho});
        in.push_back({HF_P, m.p, h->p}); in.push_back({HF_CS, m.cs, h->cs});
    }
    // mirror k is free once the compute of its last step is done
    if (c->computed_pending[k]) CUDA_TRY(cudaStreamWaitEvent(c->in_stream, c->ev_computed[k], 0));
    for (auto& q : in) {
        if (!q.hh) continue;
        for (int i = 0; i < kHostChunks; ++i) {
            // mirror k's copy-out of this piece (two steps back) and the host
            // buffer's latest write (the previous step's copy-out from mirror j)
            const int e = q.id * kHostChunks + i;
            if (c->out_pending[k][e]) CUDA_TRY(cudaStreamWaitEvent(c->in_stream, c->ev_out[k][e], 0));
            if (c->out_pending[j][e]) CUDA_TRY(cudaStreamWaitEvent(c->in_stream, c->ev_out[j][e], 0));
            const size_t a0 = piece(i), a1 = piece(i + 1);
            if (a1 > a0)
                CUDA_TRY(cudaMemcpyAsync(q.d + a0, q.hh + a0, sizeof(double) * (a1 - a0), cudaMemcpyHostToDevice,
                                         c->in_stream));
        }
    }
    CUDA_TRY(cudaEventRecord(c->ev_in, c->in_stream));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_in, 0));
    // the compute overwrites every output field of mirror k: its copy-out two
    // steps back must have finished (for the fields that are also inputs this
    // is already implied by their copy-in)
    for (int f = 0; f < HF_COUNT * kHostChunks; ++f)
        if (c->out_pending[k][f]) CUDA_TRY(cudaStreamWaitEvent(s, c->ev_out[k][f], 0));
    // leapfrog: step 0 computes the initial accelerations; later steps carry
    // the caller's g_a of the previous step
    if (c->cfg.integrator == 2) c->first_rhs_done = step != 0;
    const bool overlap = c->cfg.integrator == 2 && h->x && h->y && h->z;
    if (overlap) {
        if (!c->copy_stream) {
            CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_drift, cudaEventDisableTiming));
        }
        // the drifted positions are written to the host during this step's
        // right-hand side, after this step's copy-in has read them
        c->pos_out[0] = h->x; c->pos_out[1] = h->y; c->pos_out[2] = h->z;
    }
    int rc = integrate_step(c, &m, step, dt_out, false);
    c->pos_out[0] = c->pos_out[1] = c->pos_out[2] = nullptr;
    if (rc) return rc;
    if (overlap) {
        // the drifted positions went out on copy_stream during the RHS
        for (int f = HF_X * kHostChunks; f < (HF_Z + 1) * kHostChunks; ++f) {
            CUDA_TRY(cudaEventRecord(c->ev_out[k][f], c->copy_stream));
            c->out_pending[k][f] = true;
        }
    }
    CUDA_TRY(cudaEventRecord(c->ev_computed[k], s));
    c->computed_pending[k] = true;
    ++c->host_steps;
    CUDA_TRY(cudaStreamWaitEvent(c->out_stream, c->ev_computed[k], 0));
    std::vector<Field> outp = {{HF_VX, m.vx, h->vx}, {HF_VY, m.vy, h->vy}, {HF_VZ, m.vz, h->vz}};
    if (!overlap) {
        outp.push_back({HF_X, m.x, h->x}); outp.push_back({HF_Y, m.y, h->y}); outp.push_back({HF_Z, m.z, h->z});
    }
    if (c->cfg.gravity) {
        outp.push_back({HF_GX, m.g_ax, h->g_ax}); outp.push_back({HF_GY, m.g_ay, h->g_ay});
        outp.push_back({HF_GZ, m.g_az, h->g_az});
    }
    if (c->cfg.sph) {
        outp.push_back({HF_H, m.sml, h->sml}); outp.push_back({HF_E, m.e, h->e});
        outp.push_back({HF_RHO, m.rho, h->rho}); outp.push_back({HF_P, m.p, h->p}); outp.push_back({HF_CS, m.cs, h->cs});
        outp.push_back({HF_AX, m.ax, h->ax}); outp.push_back({HF_AY, m.ay, h->ay}); outp.push_back({HF_AZ, m.az, h->az});
    }
    for (auto& q : outp) {
        if (!q.hh) continue;
        for (int i = 0; i < kHostChunks; ++i) {
            const size_t a0 = piece(i), a1 = piece(i + 1);
            if (a1 > a0)
                CUDA_TRY(cudaMemcpyAsync(q.hh + a0, q.d + a0, sizeof(double) * (a1 - a0), cudaMemcpyDeviceToHost,
                                         c->out_stream));
            const int e = q.id * kHostChunks + i;
            CUDA_TRY(cudaEventRecord(c->ev_out[k][e], c->out_stream));
            c->out_pending[k][e] = true;
        }
    }
    return MHPC_OK;
}

int mhpc_host_wait(mhpc_ctx* c) {
    if (!c) return MHPC_ERR_ARG;
    if (c->in_stream) CUDA_TRY(cudaStreamSynchronize(c->in_stream));
    if (c->out_stream) CUDA_TRY(cudaStreamSynchronize(c->out_stream));
    if (c->copy_stream) CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return read_status(c);
}

int mhpc_integrate_host(mhpc_ctx* c, mhpc_particles* h, int step, double* dt_out) {
    TRY(mhpc_integrate_host_async(c, h, step, dt_out));
    return mhpc_host_wait(c);
}

int mhpc_export_sorted(mhpc_ctx* c, uint64_t* keys_dev, int* perm_dev) {
    if (!c) return MHPC_ERR_ARG;
    const int n = c->last_n;
    if (keys_dev) CUDA_TRY(cudaMemcpyAsync(keys_dev, c->skey, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c->stream));
    if (perm_dev) CUDA_TRY(cudaMemcpyAsync(perm_dev, c->perm, sizeof(int) * n, cudaMemcpyDeviceToDevice, c->stream));
    return read_status(c);
}

int mhpc_export_tree(mhpc_ctx* c, int num_nodes, int* child, int* level, double* x, double* y, double* z, double* m,
                     int* cells_out) {
    if (!c || !child) return MHPC_ERR_ARG;
    int code = read_status(c);
    if (code) return code;
    const int n = c->last_n;
    int total = 0;
    CUDA_TRY(cudaMemcpy(&total, c->T.nodes, sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int2> link(total);
    std::vector<int> first(total);
    std::vector<double4> com(total);
    std::vector<int> perm(n);
    std::vector<uint64_t> skey(n);
    CUDA_TRY(cudaMemcpy(link.data(), c->T.link, sizeof(int2) * total, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(first.data(), c->T.first, sizeof(int) * total, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(com.data(), c->T.com, sizeof(double4) * total, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(perm.data(), c->perm, sizeof(int) * n, cudaMemcpyDeviceToHost));
    std::vector<double> px(n), py(n), pz(n);
    CUDA_TRY(cudaMemcpy(px.data(), c->sx, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(py.data(), c->sy, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(pz.data(), c->sz, sizeof(double) * n, cudaMemcpyDeviceToHost));
    long long ord[2];
    CUDA_TRY(cudaMemcpy(ord, c->ord, sizeof(ord), cudaMemcpyDeviceToHost));
    const double lo = ord_to_dbl(ord[0]), hi = ord_to_dbl(ord[1]);
    // cell ids: n + ordinal in pre-order
    std::vector<int> id(total, -1);
    int cells = 0;
    for (int i = 0; i < total; ++i) id[i] = (link[i].y & ND_LEAF) ? perm[first[i]] : n + cells++;
    if (cells_out) *cells_out = cells;
    if (n + cells > num_nodes) return MHPC_ERR_CAPACITY;
    for (long i = 0; i < 8L * num_nodes; ++i) child[i] = -1;
    if (level) for (int i = 0; i < num_nodes; ++i) level[i] = -1;
    // octant of a sorted particle at level L (1-based), reference bit rule
    auto octant = [&](int sidx, int L) {
        double mn[3] = {lo, lo, lo}, mx[3] = {hi, hi, hi};
        double p[3] = {px[sidx], py[sidx], pz[sidx]};
        int son = 0;
        for (int l = 0; l < L; ++l) {
            son = 0;
            for (int d = 0; d < 3; ++d) {
                volatile double mid = 0.5 * (mn[d] + mx[d]);
                if (p[d] < mid) { son += 1 << d; mx[d] = mid; } else mn[d] = mid;
            }
        }
        return son;
    };
    for (int i = 0; i < total; ++i) {
        const int L = link[i].y & 0xff;
        const int self = id[i];
        if (level) level[self] = L;
        if (!(link[i].y & ND_LEAF)) {
            if (x) x[self] = com[i].x;
            if (y) y[self] = com[i].y;
            if (z) z[self] = com[i].z;
            if (m) m[self] = com[i].w;
            for (int ch = i + 1; ch < link[i].x; ch = link[ch].x) {
                const int slot = octant(first[ch], L + 1);
                child[8 * self + slot] = id[ch];
            }
        }
        if (L == 1) child[octant(first[i], 1)] = self;
    }
    return MHPC_OK;
}

int mhpc_get_stats(mhpc_ctx* c, mhpc_stats* o) {
    if (!c || !o) return MHPC_ERR_ARG;
    std::memset(o, 0, sizeof(*o));
    int code = read_status(c);
    o->n = c->last_n;
    if (c->last_n > 0) {
        int total = 0;
        CUDA_TRY(cudaMemcpy(&total, c->T.nodes, sizeof(int), cudaMemcpyDeviceToHost));
        o->cells = total - c->last_n;
        CUDA_TRY(cudaMemcpy(o->bbox, c->bbox, sizeof(double) * 6, cudaMemcpyDeviceToHost));
        o->radius = 0.5 * (o->bbox[1] - o->bbox[0]);
    }
    DevStatus& h = *c->h_st;
    o->max_level = h.max_level;
    o->key_collisions = h.key_collisions;
    o->gravity_interactions = (double)h.interactions;
    o->gravity_nodes_visited = (double)h.nodes_visited;
    o->gravity_quad_interactions = (double)h.quad_interactions;
    o->max_noi = h.max_noi;
    o->mean_noi = c->last_n > 0 ? (double)h.noi_sum / c->last_n : 0.0;
    o->sml_out_of_band = h.sml_out_of_band;
    o->predictor_used = h.predictor_used;
    o->predictor_fallback = h.predictor_fallback;
    o->sml_band_before = c->band_ran ? h.sml_band_before : -1;
    o->sml_band_skipped = h.sml_band_skipped;
    RunTotals R;
    CUDA_TRY(cudaMemcpy(&R, c->run, sizeof(R), cudaMemcpyDeviceToHost));
    if (c->st_pending) {  // the last RHS, not yet folded on the device
        const unsigned long long oob = (unsigned long long)(h.sml_out_of_band > 0 ? h.sml_out_of_band : 0);
        R.rhs += 1;
        R.oob_sum += oob;
        R.oob_max = oob > R.oob_max ? oob : R.oob_max;
        if (c->band_ran && h.sml_band_before >= 0) {
            R.before_sum += (unsigned long long)h.sml_band_before;
            R.band_rhs += 1;
        }
        R.used_sum += (unsigned long long)(h.predictor_used > 0 ? h.predictor_used : 0);
        R.fallback_sum += (unsigned long long)(h.predictor_fallback > 0 ? h.predictor_fallback : 0);
    }
    o->run_rhs = (int)R.rhs;
    o->run_out_of_band_max = (int)R.oob_max;
    o->run_out_of_band_sum = (double)R.oob_sum;
    o->run_band_before_sum = (double)R.before_sum;
    o->run_band_rhs = (int)R.band_rhs;
    o->run_predictor_used_sum = (double)R.used_sum;
    o->run_predictor_fallback_sum = (double)R.fallback_sum;
    const int pairs[12][2] = {{EV_START, EV_KEYS}, {EV_KEYS, EV_SORT}, {EV_SORT, EV_TREE},  {EV_TREE, EV_COM},
                              {EV_COM, EV_GRAV},   {EV_SML, EV_LISTS}, {EV_COM, EV_SML},    {EV_FRNN, EV_DENS},
                              {EV_DENS, EV_FORCES}, {EV_LISTS, EV_FRNN}, {-1, -1},          {EV_START, EV_END}};
    for (int k = 0; k < 12; ++k) {
        int a = pairs[k][0], b = pairs[k][1];
        if (a >= 0 && c->ev_recorded[a] && c->ev_recorded[b]) cudaEventElapsedTime(&o->ms_stage[k], c->ev[a], c->ev[b]);
    }
    if (c->ev_recorded[EV_GRAV] && c->ev_recorded[EV_SML]) {
        // gravity ran before SPH: the SML stage starts at EV_GRAV
        cudaEventElapsedTime(&o->ms_stage[6], c->ev[EV_GRAV], c->ev[EV_SML]);
    }
    return code;
}

int mhpc_stats_reset_run(mhpc_ctx* c) {
    if (!c) return MHPC_ERR_ARG;
    CUDA_TRY(cudaMemsetAsync(c->run, 0, sizeof(RunTotals), c->stream));
    c->st_pending = false;
    return MHPC_OK;
}

int mhpc_remove_particles(mhpc_ctx* c, mhpc_particles* p, int* n_removed) {
    if (!c || !p) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    if (n_removed) *n_removed = 0;
    const int n = p->n;
    if (n == 0) return MHPC_OK;
    const int crit = c->cfg.remove_particles_criterion;
    if (crit != 0 && crit != 1) return MHPC_ERR_CONFIG;
    cudaStream_t s = c->stream;
    // the tree's per-position scratch (free between right-hand sides) holds
    // the flags and their exclusive scan; the sorted-copy buffers hold the
    // compacted arrays before they are copied back
    int* keep = c->T.cnt;
    int* rank = c->T.off;
    TRY(launch_remove_mark(n, p->x, p->y, p->z, crit, c->cfg.remove_particles_dimension, keep, s));
    TRY(scan_exclusive_i32(keep, rank, n, c->scan_scratch, s));
    int kept = 0;
    CUDA_TRY(cudaMemcpyAsync(&kept, rank + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (kept == n) return MHPC_OK;
    double* dfields[] = {p->x, p->y, p->z, p->mass, p->vx, p->vy, p->vz, p->ax, p->ay, p->az,
                         p->g_ax, p->g_ay, p->g_az, p->g_ax_old, p->g_ay_old, p->g_az_old,
                         p->sml, p->rho, p->p, p->cs, p->e, p->drhodt, p->dedt, p->dsmldt};
    for (double* f : dfields) {
        if (!f) continue;
        TRY(launch_compact_d(n, keep, rank, f, c->sx, s));
        CUDA_TRY(cudaMemcpyAsync(f, c->sx, sizeof(double) * (size_t)kept, cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(cudaMemsetAsync(f + kept, 0, sizeof(double) * (size_t)(n - kept), s));
    }
    int* ifields[] = {p->noi, p->material_id};
    for (int* f : ifields) {
        if (!f) continue;
        TRY(launch_compact_i(n, keep, rank, f, c->T.leaf_node, s));
        CUDA_TRY(cudaMemcpyAsync(f, c->T.leaf_node, sizeof(int) * (size_t)kept, cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(cudaMemsetAsync(f + kept, 0, sizeof(int) * (size_t)(n - kept), s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    p->n = kept;
    c->grav_prev_n = -1;  // the previous accelerations no longer match the particle count
    if (n_removed) *n_removed = n - kept;
    return MHPC_OK;
}

int mhpc_diagnostics(mhpc_ctx* c, const mhpc_particles* p, double* out) {
    if (!c || !p || !out) return MHPC_ERR_ARG;
    TRY(check_particles(c, p));
    TRY(launch_diagnostics(*p, c->cfg.sph, c->diag_part, c->diag_out, c->stream));
    CUDA_TRY(cudaMemcpyAsync(out, c->diag_out, sizeof(double) * 11, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MHPC_OK;
}

int mhpc_potential(mhpc_ctx* c, const mhpc_particles* p, double* pot_dev, double* energy_out) {
    if (!c || !p) return MHPC_ERR_ARG;
    if (!c->cfg.gravity) return MHPC_ERR_CONFIG;
    TRY(check_particles(c, p));
    const int n = p->n;
    if (n == 0) {
        if (energy_out) *energy_out = 0.0;
        return MHPC_OK;
    }
    cudaStream_t s = c->stream;
    if (!c->pot_scratch) return MHPC_ERR_ARG;
    double* pot = pot_dev ? pot_dev : c->pot_scratch;
    double* acc = c->pot_scratch + c->cap;  // accelerations of this walk (not the caller's g_a)
    TRY(reset_status(c, s));
    c->force_wrec = true;
    const int rc = stage_tree(c, p);
    c->force_wrec = false;
    TRY(rc);
    GravParams G;
    std::memset(&G, 0, sizeof(G));
    G.n = n;
    G.eps2 = c->cfg.smoothing;
    G.h_factor = h_softening(c->cfg) ? c->cfg.softening_h_factor : 0.0;
    G.G = c->cfg.si_units ? 6.67430e-11 : 1.0;
    G.ord = c->ord;
    G.theta = c->cfg.theta_mixed;  // geometric rule: the same opening rule at every call
    G.pot = pot;
    TRY(gravity_lists(c->T, G, c->sx, c->sy, c->sz, c->sh, c->perm, acc, acc + c->cap, acc + 2 * (size_t)c->cap,
                      c->st, s));
    if (energy_out) {
        TRY(launch_potential_energy(n, p->mass, pot, c->diag_part, c->diag_out, s));
        CUDA_TRY(cudaMemcpyAsync(energy_out, c->diag_out, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    return read_status(c);
}

int mhpc_direct_gravity(const double* x, const double* y, const double* z, const double* m, int n, const int* targets,
                        int nt, double eps2, double* gax, double* gay, double* gaz, void* stream) {
    if (n < 0 || nt < 0 || (nt > 0 && (!x || !y || !z || !m || !targets || !gax || !gay || !gaz))) return MHPC_ERR_ARG;
    return launch_direct(x, y, z, m, n, targets, nt, eps2, nullptr, gax, gay, gaz, (cudaStream_t)stream);
}

int mhpc_direct_gravity_soft(const double* x, const double* y, const double* z, const double* m, int n,
                             const int* targets, int nt, double eps2, const double* eps2_targets, double* gax,
                             double* gay, double* gaz, void* stream) {
    if (n < 0 || nt < 0 || (nt > 0 && (!x || !y || !z || !m || !targets || !eps2_targets || !gax || !gay || !gaz)))
        return MHPC_ERR_ARG;
    return launch_direct(x, y, z, m, n, targets, nt, eps2, eps2_targets, gax, gay, gaz, (cudaStream_t)stream);
}

// ------------------------------------------------ learned smoothing length
int mhpc_mlp_num_params(void) { return MLP_NPARAM; }

int mhpc_mlp_reset(mhpc_ctx* c, uint64_t seed) {
    if (!c || !c->mlp) return MHPC_ERR_ARG;
    return mlp_reset(c->mlp, seed, c->stream);
}

int mhpc_mlp_train(mhpc_ctx* c, int iters, float lr, float* loss_out) {
    if (!c || !c->mlp || iters < 0 || !(lr > 0.f)) return MHPC_ERR_ARG;
    return mlp_train(c->mlp, iters, lr, 8192, loss_out, c->stream);
}

int mhpc_mlp_forward_backward(mhpc_ctx* c, const float* feats, int rows, const float* target, float* out, float* grad,
                              float* loss_out) {
    if (!c || !c->mlp || !feats || !target || rows <= 0) return MHPC_ERR_ARG;
    return mlp_forward_backward(c->mlp, feats, rows, target, out, grad, loss_out, c->stream);
}

int mhpc_mlp_get_params(mhpc_ctx* c, float* host) {
    if (!c || !c->mlp || !host) return MHPC_ERR_ARG;
    return mlp_get_params(c->mlp, host, c->stream);
}

int mhpc_mlp_set_params(mhpc_ctx* c, const float* host) {
    if (!c || !c->mlp || !host) return MHPC_ERR_ARG;
    return mlp_set_params(c->mlp, host, c->stream);
}

}  // extern "C"
