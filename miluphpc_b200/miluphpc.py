"""Host-side mirror of milupHPC's RHS interface on top of libmhpc.

`Miluphpc` plays the role of the reference class of the same name
(include/miluphpc.h): it owns the particle SoA on the device, exposes
`rhs(step, self_gravity)` (Miluphpc::rhs, include/miluphpc.h:478) and
`integrate(step)` (the integrators' virtual integrate(int step),
include/miluphpc.h:485).  All compute goes through the C ABI of libmhpc;
torch only provides device memory and the CUDA stream.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import Config, Material, Particles, Stats, check

DOUBLE_FIELDS = _lib.PARTICLE_DOUBLE_FIELDS


def config_from_info(path):
    cfg = _lib.default_config()
    check(_lib.load().mhpc_config_from_info(str(path).encode(), ctypes.byref(cfg)), "config_from_info")
    return cfg


def materials_from_cfg(path, cap=8):
    arr = (Material * cap)()
    cnt = ctypes.c_int(0)
    check(_lib.load().mhpc_materials_from_cfg(str(path).encode(), arr, cap, ctypes.byref(cnt)),
          "materials_from_cfg")
    return [arr[i] for i in range(cnt.value)]


def material(interactions=60, sml=0.0, alpha=1.0, beta=2.0, eos_type=9, K=0.0, gamma=5.0 / 3.0):
    m = Material()
    m.id = 0
    m.interactions = interactions
    m.sml = sml
    m.alpha = alpha
    m.beta = beta
    m.eos_type = eos_type
    m.polytropic_K = K
    m.polytropic_gamma = gamma
    return m


class Miluphpc:
    """Particles on one GPU plus a libmhpc context."""

    def __init__(self, cfg, state, materials=None, capacity=None, device="cuda:0", want_nnl=False,
                 num_nodes=None):
        self.L = _lib.load()
        self.cfg = cfg
        self.device = torch.device(device)
        n = int(len(state["x"]))
        self.n = n
        self.capacity = int(capacity or n)
        self.num_nodes = int(num_nodes or n)
        mats = materials or [material()]
        self.materials = list(mats)
        self._mats = (Material * max(1, len(mats)))(*mats)
        self.t = {}
        for f in DOUBLE_FIELDS:
            size = self.num_nodes if f in ("x", "y", "z", "mass") else n
            arr = torch.zeros(size, dtype=torch.float64, device=self.device)
            if f in state:
                arr[:n] = torch.as_tensor(np.asarray(state[f], dtype=np.float64), device=self.device)
            self.t[f] = arr
        if "sml" not in state and len(mats) and mats[0].sml > 0:
            self.t["sml"].fill_(mats[0].sml)
        self.t["noi"] = torch.zeros(n, dtype=torch.int32, device=self.device)
        if want_nnl:
            self.t["nnl"] = torch.full((n * cfg.max_num_interactions,), -1, dtype=torch.int32, device=self.device)
        if "material_id" in state:
            self.t["material_id"] = torch.as_tensor(np.asarray(state["material_id"], dtype=np.int32),
                                                    device=self.device)
        ctx = ctypes.c_void_p()
        check(self.L.mhpc_ctx_create(ctypes.byref(ctx), self.capacity, ctypes.byref(cfg), self._mats, len(mats)),
              "ctx_create")
        self.ctx = ctx
        self.stream = torch.cuda.current_stream(self.device)
        check(self.L.mhpc_ctx_set_stream(self.ctx, ctypes.c_void_p(self.stream.cuda_stream)), "set_stream")
        self._soa = self._make_soa()

    def _make_soa(self):
        p = Particles()
        p.n = self.n
        p.num_nodes = self.num_nodes
        for f in DOUBLE_FIELDS:
            setattr(p, f, ctypes.cast(ctypes.c_void_p(self.t[f].data_ptr()), _lib.P_d))
        for f in _lib.PARTICLE_INT_FIELDS:
            if f in self.t:
                setattr(p, f, ctypes.cast(ctypes.c_void_p(self.t[f].data_ptr()), _lib.P_i))
        return p

    @property
    def soa(self):
        return self._soa

    def set_config(self, cfg):
        check(self.L.mhpc_ctx_set_config(self.ctx, ctypes.byref(cfg)), "set_config")
        self.cfg = cfg

    def rhs(self, step=0, self_gravity=True):
        ms = ctypes.c_float(0)
        check(self.L.mhpc_rhs(self.ctx, ctypes.byref(self._soa), int(step), int(bool(self_gravity)),
                              ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(ms)), "rhs")
        return ms.value

    def rhs_async(self, step=0, self_gravity=True):
        check(self.L.mhpc_rhs_async(self.ctx, ctypes.byref(self._soa), int(step), int(bool(self_gravity))),
              "rhs_async")

    def status(self):
        return self.L.mhpc_ctx_status(self.ctx)

    def remove_particles(self):
        """Miluphpc::removeParticles: drop the particles outside the configured
        region (compacting every array, lowering n); returns how many left."""
        k = ctypes.c_int(0)
        check(self.L.mhpc_remove_particles(self.ctx, ctypes.byref(self._soa), ctypes.byref(k)), "remove_particles")
        self.n = self._soa.n
        return k.value

    def integrate(self, step):
        # the reference's integrators remove particles at the start of a step
        if self.cfg.remove_particles:
            self.remove_particles()
        dt = ctypes.c_double(0)
        check(self.L.mhpc_integrate(self.ctx, ctypes.byref(self._soa), int(step), ctypes.byref(dt)), "integrate")
        return dt.value

    def stats(self):
        s = Stats()
        check(self.L.mhpc_get_stats(self.ctx, ctypes.byref(s)), "stats")
        d = {f: getattr(s, f) for f, _ in Stats._fields_ if f not in ("bbox", "ms_stage")}
        d["bbox"] = list(s.bbox)
        d["ms_stage"] = dict(zip(_lib.STAGES, list(s.ms_stage)))
        return d

    def reset_run_stats(self):
        """Restart the run totals (run_* fields of stats())."""
        check(self.L.mhpc_stats_reset_run(self.ctx), "stats_reset_run")

    def diagnostics(self):
        out = (ctypes.c_double * 11)()
        check(self.L.mhpc_diagnostics(self.ctx, ctypes.byref(self._soa), out), "diagnostics")
        v = list(out)
        return dict(kinetic=v[0], internal=v[1], momentum=v[2:5], angular_momentum=v[5:8], com=v[8:11])

    def potential(self, per_particle=False):
        """Potential energy W = 1/2 sum m phi of the current positions (and, with
        per_particle, the potential phi_i as a device tensor in particle order)."""
        w = ctypes.c_double(0.0)
        pot = torch.zeros(self.n, dtype=torch.float64, device=self.device) if per_particle else None
        check(self.L.mhpc_potential(self.ctx, ctypes.byref(self._soa),
                                    ctypes.c_void_p(pot.data_ptr()) if pot is not None else None,
                                    ctypes.byref(w)), "potential")
        return (w.value, pot) if per_particle else w.value

    def export_sorted(self):
        keys = torch.zeros(self.n, dtype=torch.int64, device=self.device)
        perm = torch.zeros(self.n, dtype=torch.int32, device=self.device)
        check(self.L.mhpc_export_sorted(self.ctx, ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(perm.data_ptr())),
              "export_sorted")
        return keys.cpu().numpy().view(np.uint64), perm.cpu().numpy()

    def export_tree(self, num_nodes=None):
        nn = int(num_nodes or (2 * self.n + 20000))
        child = np.zeros(8 * nn, dtype=np.int32)
        level = np.zeros(nn, dtype=np.int32)
        x = np.zeros(nn); y = np.zeros(nn); z = np.zeros(nn); m = np.zeros(nn)
        cells = ctypes.c_int(0)
        pd = lambda a: a.ctypes.data_as(_lib.P_d)
        check(self.L.mhpc_export_tree(self.ctx, nn, child.ctypes.data_as(_lib.P_i), level.ctypes.data_as(_lib.P_i),
                                      pd(x), pd(y), pd(z), pd(m), ctypes.byref(cells)), "export_tree")
        return dict(child=child, level=level, x=x, y=y, z=z, m=m, cells=cells.value, num_nodes=nn)

    def numpy(self, f):
        return self.t[f][: self.n].cpu().numpy()

    def close(self):
        if getattr(self, "ctx", None):
            self.L.mhpc_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def direct_gravity(x, y, z, m, targets, eps2, eps2_targets=None):
    """FP64 direct summation on the GPU (verification): torch tensors in, (gx, gy, gz) out.
    eps2_targets (optional, per target) is added to eps2 (h-tied softening)."""
    L = _lib.load()
    nt = int(targets.numel())
    out = [torch.zeros(nt, dtype=torch.float64, device=x.device) for _ in range(3)]
    st = torch.cuda.current_stream(x.device).cuda_stream
    ptrs = [ctypes.c_void_p(t.data_ptr()) for t in (x, y, z, m)]
    if eps2_targets is None:
        check(L.mhpc_direct_gravity(*ptrs, int(x.numel()), ctypes.c_void_p(targets.data_ptr()), nt, float(eps2),
                                    *(ctypes.c_void_p(o.data_ptr()) for o in out), ctypes.c_void_p(st)),
              "direct_gravity")
    else:
        check(L.mhpc_direct_gravity_soft(*ptrs, int(x.numel()), ctypes.c_void_p(targets.data_ptr()), nt,
                                         float(eps2), ctypes.c_void_p(eps2_targets.data_ptr()),
                                         *(ctypes.c_void_p(o.data_ptr()) for o in out), ctypes.c_void_p(st)),
              "direct_gravity_soft")
    return out
