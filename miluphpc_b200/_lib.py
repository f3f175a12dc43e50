"""ctypes binding of libmhpc.so (declared in include/mhpc.h).

The library is the only compute path: if it is missing or fails to load this
module raises, there is no Python or CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MHPC_LIBRARY") or os.path.join(HERE, "libmhpc.so")

c_int, c_double, c_float, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p
P_d = ctypes.POINTER(ctypes.c_double)
P_i = ctypes.POINTER(ctypes.c_int)
P_u64 = ctypes.POINTER(ctypes.c_uint64)
P_f = ctypes.POINTER(ctypes.c_float)

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA runtime error", 3: "capacity", 4: "node pool exhausted",
    5: "depth exceeded", 6: "too many neighbours", 7: "non-finite position or density", 8: "config error",
    9: "no CUDA device", 10: "bounded device wait ran out", 11: "unsupported option",
}


class MhpcError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        super().__init__("%s: mhpc status %d (%s)" % (where, code, STATUS.get(code, "?")))


class Config(ctypes.Structure):
    """mhpc_config (run-time SimulationParameters + parameter.h switches)."""
    _fields_ = [
        ("integrator", c_int), ("time_step", c_double), ("max_time_step", c_double), ("time_end", c_double),
        ("sfc", c_int), ("theta", c_double), ("smoothing", c_double), ("smoothing_kernel", c_int),
        ("gravity_force_version", c_int), ("sph_frnn_version", c_int), ("calculate_energy", c_int),
        ("calculate_angular_momentum", c_int), ("calculate_center_of_mass", c_int), ("remove_particles", c_int),
        ("remove_particles_criterion", c_int), ("remove_particles_dimension", c_double),
        ("gravity", c_int), ("sph", c_int), ("integrate_energy", c_int), ("integrate_density", c_int),
        ("integrate_sml", c_int), ("variable_sml", c_int), ("si_units", c_int), ("max_num_interactions", c_int),
        ("nb_tolerance", c_int), ("max_sml_iterations", c_int),
        ("precision", c_int), ("theta_mixed", c_double), ("learned_h", c_int), ("softening_mode", c_int),
        ("softening_h_factor", c_double), ("node_pool_factor", c_double),
        ("gravity_mac", c_int), ("mac_alpha", c_double), ("balsara", c_int), ("mac_quad_alpha", c_double),
        ("sml_band_rounds", c_int), ("learned_refresh_every", c_int), ("learned_refresh_iters", c_int),
    ]


class Material(ctypes.Structure):
    """mhpc_material (include/materials/material.cuh:123-150 of the reference)."""
    _fields_ = [
        ("id", c_int), ("interactions", c_int), ("sml", c_double), ("alpha", c_double), ("beta", c_double),
        ("eos_type", c_int), ("polytropic_K", c_double), ("polytropic_gamma", c_double), ("rho_0", c_double),
        ("bulk_modulus", c_double), ("n", c_double), ("shear_modulus", c_double),
    ]


PARTICLE_DOUBLE_FIELDS = ["x", "y", "z", "mass", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay", "g_az",
                          "g_ax_old", "g_ay_old", "g_az_old", "sml", "rho", "p", "cs", "e", "drhodt", "dedt",
                          "dsmldt"]
PARTICLE_INT_FIELDS = ["noi", "nnl", "material_id", "level"]


class Particles(ctypes.Structure):
    """mhpc_particles: the Particles SoA of pointers."""
    _fields_ = [("n", c_int), ("num_nodes", c_int)] + [(f, P_d) for f in PARTICLE_DOUBLE_FIELDS] + \
               [(f, P_i) for f in PARTICLE_INT_FIELDS]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n", c_int), ("cells", c_int), ("max_level", c_int), ("key_collisions", c_int),
        ("bbox", c_double * 6), ("radius", c_double), ("gravity_interactions", c_double),
        ("gravity_nodes_visited", c_double), ("gravity_quad_interactions", c_double), ("max_noi", c_int), ("mean_noi", c_double),
        ("sml_sweeps", c_int), ("sml_out_of_band", c_int), ("predictor_used", c_int),
        ("predictor_fallback", c_int), ("ms_stage", c_float * 12), ("sml_band_before", c_int),
        ("sml_band_skipped", c_int),
        ("run_rhs", c_int), ("run_out_of_band_max", c_int), ("run_out_of_band_sum", c_double),
        ("run_band_before_sum", c_double), ("run_band_rhs", c_int), ("run_pad", c_int),
        ("run_predictor_used_sum", c_double), ("run_predictor_fallback_sum", c_double),
    ]


STAGES = ["bbox_keys", "sort", "tree", "com", "gravity", "frnn", "sml", "density", "forces", "band", "unused",
          "total"]

_lib = None


def load():
    """Load libmhpc.so; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libmhpc.so not built (run __graft_entry__.build() or python miluphpc_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    L.mhpc_status_string.restype = ctypes.c_char_p
    L.mhpc_status_string.argtypes = [c_int]
    L.mhpc_version.restype = c_int
    L.mhpc_config_default.argtypes = [ctypes.POINTER(Config)]
    L.mhpc_config_default.restype = None
    L.mhpc_config_from_info.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config)]
    L.mhpc_materials_from_cfg.argtypes = [ctypes.c_char_p, ctypes.POINTER(Material), c_int, P_i]
    L.mhpc_bbox.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    L.mhpc_keys.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]
    L.mhpc_sort_scratch_bytes.argtypes = [c_int]
    L.mhpc_sort_scratch_bytes.restype = ctypes.c_size_t
    L.mhpc_sort_pairs.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, ctypes.c_size_t,
                                  c_void_p]
    L.mhpc_sort_noalloc_max_n.restype = c_int
    L.mhpc_sort_pairs_noalloc.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    L.mhpc_ctx_create.argtypes = [ctypes.POINTER(c_void_p), c_int, ctypes.POINTER(Config),
                                  ctypes.POINTER(Material), c_int]
    L.mhpc_ctx_destroy.argtypes = [c_void_p]
    L.mhpc_ctx_set_stream.argtypes = [c_void_p, c_void_p]
    L.mhpc_ctx_set_config.argtypes = [c_void_p, ctypes.POINTER(Config)]
    L.mhpc_rhs.argtypes = [c_void_p, ctypes.POINTER(Particles), c_int, c_int, c_void_p, P_f]
    L.mhpc_rhs_async.argtypes = [c_void_p, ctypes.POINTER(Particles), c_int, c_int]
    L.mhpc_ctx_status.argtypes = [c_void_p]
    L.mhpc_integrate.argtypes = [c_void_p, ctypes.POINTER(Particles), c_int, P_d]
    L.mhpc_integrate_host.argtypes = [c_void_p, ctypes.POINTER(Particles), c_int, P_d]
    L.mhpc_integrate_host_async.argtypes = [c_void_p, ctypes.POINTER(Particles), c_int, P_d]
    L.mhpc_host_wait.argtypes = [c_void_p]
    L.mhpc_stage_tree.argtypes = [c_void_p, ctypes.POINTER(Particles)]
    L.mhpc_stage_gravity.argtypes = [c_void_p, ctypes.POINTER(Particles)]
    L.mhpc_stage_sph.argtypes = [c_void_p, ctypes.POINTER(Particles)]
    PP = ctypes.POINTER(Particles)
    for f in ("mhpc_tree_build", "mhpc_com", "mhpc_density_eos", "mhpc_forces"):
        getattr(L, f).argtypes = [c_void_p, PP]
    L.mhpc_gravity.argtypes = [c_void_p, PP, c_int]
    L.mhpc_frnn.argtypes = [c_void_p, PP, c_int, c_int]
    L.mhpc_integrate_leapfrog.argtypes = [c_void_p, PP, c_double, c_int]
    L.mhpc_integrate_euler.argtypes = [c_void_p, PP, c_double]
    L.mhpc_integrate_pc_step_size.argtypes = [c_void_p, PP, c_double, c_void_p]
    L.mhpc_integrate_pc_predictor.argtypes = [c_void_p, PP, PP, c_void_p]
    L.mhpc_integrate_pc_corrector.argtypes = [c_void_p, PP, PP, c_void_p]
    L.mhpc_export_sorted.argtypes = [c_void_p, c_void_p, c_void_p]
    L.mhpc_export_tree.argtypes = [c_void_p, c_int, P_i, P_i, P_d, P_d, P_d, P_d, P_i]
    L.mhpc_get_stats.argtypes = [c_void_p, ctypes.POINTER(Stats)]
    L.mhpc_stats_reset_run.argtypes = [c_void_p]
    L.mhpc_diagnostics.argtypes = [c_void_p, ctypes.POINTER(Particles), P_d]
    L.mhpc_potential.argtypes = [c_void_p, ctypes.POINTER(Particles), c_void_p, P_d]
    L.mhpc_remove_particles.argtypes = [c_void_p, ctypes.POINTER(Particles), P_i]
    L.mhpc_direct_gravity.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_double,
                                      c_void_p, c_void_p, c_void_p, c_void_p]
    L.mhpc_direct_gravity_soft.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                           c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    L.mhpc_fp32_peak.argtypes = [P_d]
    L.mhpc_mlp_reset.argtypes = [c_void_p, ctypes.c_uint64]
    L.mhpc_mlp_train.argtypes = [c_void_p, c_int, c_float, P_f]
    L.mhpc_mlp_num_params.restype = c_int
    L.mhpc_mlp_forward_backward.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, P_f]
    L.mhpc_mlp_get_params.argtypes = [c_void_p, P_f]
    L.mhpc_mlp_set_params.argtypes = [c_void_p, P_f]
    _lib = L
    return L


def check(code, where=""):
    if code != 0:
        raise MhpcError(code, where)


def default_config(**kw):
    cfg = Config()
    load().mhpc_config_default(ctypes.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise AttributeError(k)
        setattr(cfg, k, v)
    return cfg


# Exported symbols declared in include/mhpc.h (checked by the CPU tests).
EXPORTS = [
    "mhpc_status_string", "mhpc_version", "mhpc_config_default", "mhpc_config_from_info",
    "mhpc_materials_from_cfg", "mhpc_bbox", "mhpc_keys", "mhpc_sort_scratch_bytes", "mhpc_sort_pairs",
    "mhpc_sort_noalloc_max_n", "mhpc_sort_pairs_noalloc",
    "mhpc_ctx_create", "mhpc_ctx_destroy", "mhpc_ctx_set_stream", "mhpc_ctx_set_config", "mhpc_rhs",
    "mhpc_rhs_async", "mhpc_ctx_status", "mhpc_integrate", "mhpc_integrate_host", "mhpc_stage_tree",
    "mhpc_stage_gravity", "mhpc_stage_sph", "mhpc_export_sorted", "mhpc_export_tree", "mhpc_get_stats",
    "mhpc_diagnostics", "mhpc_potential", "mhpc_direct_gravity", "mhpc_fp32_peak", "mhpc_mlp_reset", "mhpc_mlp_train", "mhpc_mlp_num_params",
    "mhpc_mlp_forward_backward", "mhpc_mlp_get_params", "mhpc_mlp_set_params",
    "mhpc_remove_particles", "mhpc_direct_gravity_soft",
    "mhpc_tree_build", "mhpc_com", "mhpc_gravity", "mhpc_frnn", "mhpc_density_eos", "mhpc_forces",
    "mhpc_integrate_leapfrog", "mhpc_integrate_euler", "mhpc_integrate_pc_step_size",
    "mhpc_integrate_pc_predictor", "mhpc_integrate_pc_corrector", "mhpc_stats_reset_run",
    "mhpc_integrate_host_async", "mhpc_host_wait",
]
