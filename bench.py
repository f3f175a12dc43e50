#!/usr/bin/env python
"""Particle-steps/s of milupHPC's right-hand side + integrator on one B200.

A step is one integration step (RHS: bounding box, keys, radix sort, tree,
centres of mass / multipoles, Barnes-Hut walk; plus the FP64 leapfrog update)
over the workload's synthetic particles, which stay resident in HBM.  The
default workload is the 16.7M-particle Plummer sphere (Hilbert keys, leapfrog
dt = 0.01, eps = 0.01) run with the mixed-precision walk at the opening
parameter that meets p99 relative force error <= 1e-3 against FP64 direct
summation.  `--impl reference` times the reference algorithm (FP64,
computeForces_v2 semantics, at the opening parameter that meets the same
error bar) as restated by the CPU oracle on the host cores.

Multi-GPU (torchrun, one process per GPU): replicas only — every rank runs
an independent copy of the workload; time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # Plummer at scale, precision form: N = 2^24, Hilbert keys, leapfrog dt 0.01
    # (plain FP64 v2 at theta 0.15: p99 7.5e-4 against the mixed run's 8.0e-4)
    "plummer16m": dict(kind="gravity", n=1 << 24, sfc=1, dt=0.01, eps2=1e-4, theta=0.5, theta_mixed=0.28,
                       mac_alpha=1.8e-3, mac_quad_alpha=3e-4, theta_plain_matched=0.15, seed=1, drift_steps=50),
    # profiling case of the walk: node data (~190 MB) larger than L2
    "plummer2m": dict(kind="gravity", n=1 << 21, sfc=1, dt=0.01, eps2=1e-4, theta=0.5, theta_mixed=0.28,
                      mac_alpha=1.8e-3, mac_quad_alpha=3e-4, theta_plain_matched=0.15, seed=1, drift_steps=50),
    # Sedov blast, SPH only: 128^3 lattice, fixed h = 2.5 dx, predictor-corrector
    "sedov2m": dict(kind="sph", nside=128, n=128 ** 3, sfc=0, dt_max=1e-4, seed=2),
    "sedov262k": dict(kind="sph", nside=64, n=64 ** 3, sfc=0, dt_max=1e-4, seed=2),
    # self-gravitating isothermal rotating cloud, variable h (60 +- 5), learned h
    # (accuracy-matched on the cloud with h-tied softening, p99 <= 1e-3 against the
    # direct sum softened with the h the walk used: mixed relative rule alpha = 1.0e-3
    # -> 8.1e-4 at 1M, 1.5e-3 at 8.4M (1.2e-3 -> 8.2e-4, 1.8e-3 -> 9.7e-4); plain
    # FP64 v2 theta = 0.05 -> 9.7e-4 at 1M, theta = 0.07 -> 2.9e-3 at 8.4M)
    "cloud1m": dict(kind="cloud", n=1 << 20, sfc=1, dt=0.002, theta=0.5, theta_mixed=0.25, mac_alpha=1.0e-3,
                    theta_plain_matched=0.05, train_steps=20, train_iters=1500, seed=3),
    "cloud8m": dict(kind="cloud", n=1 << 23, sfc=1, dt=0.002, theta=0.6, theta_mixed=0.25, mac_alpha=1.5e-3,
                    theta_plain_matched=0.05, train_steps=20, train_iters=1500, seed=3),
    # the reference's own single-rank case: N = 131072, Lebesgue, leapfrog dt 0.025
    "plummer131k": dict(kind="gravity", n=131072, sfc=0, dt=0.025, eps2=1e-4, theta=0.5, theta_mixed=0.28,
                        mac_alpha=1.8e-3, mac_quad_alpha=3e-4, theta_plain_matched=0.15, seed=1, drift_steps=10),
}

FLOP_MONO = 19   # flop per accepted particle-node monopole interaction
FLOP_QUAD = 34   # extra flop of the quadrupole term of an accepted cell


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def job_rate(ms_local, n_per_rank, steps, world, device):
    """Whole-job particle-steps/s of `world` replicas of n_per_rank particles:
    the slowest replica's device time (max over ranks) bounds the job.
    Returns (value, max ms); every rank takes part in the reduction."""
    import torch
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return n_per_rank * world * steps / (ms_max / 1e3), ms_max


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [a.strip() for a in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp32_peak_tflops(torch):
    """Measured FP32 FMA throughput of this GPU (CUDA cores): libmhpc's own
    dependent-FMA kernel, best of 3, used as the gravity walk's roofline."""
    from miluphpc_b200 import _lib
    import ctypes
    L = _lib.load()
    best = 0.0
    for _ in range(3):
        t = ctypes.c_double(0)
        _lib.check(L.mhpc_fp32_peak(ctypes.byref(t)), "fp32_peak")
        best = max(best, t.value)
    return best


def plummer_state(wl, rank):
    from miluphpc_b200 import ics
    if wl["kind"] == "sph":
        S = ics.sedov(nside=wl["nside"], seed=wl["seed"] + 1000 * rank)
        S["p"] = np.zeros(len(S["x"]))
        S["cs"] = np.zeros(len(S["x"]))
        return S
    if wl["kind"] == "cloud":
        C = ics.rotating_cloud(wl["n"], seed=wl["seed"] + 1000 * rank)
        C["p"] = np.zeros(wl["n"])
        C["cs"] = np.zeros(wl["n"])
        return C
    return ics.plummer(wl["n"], seed=wl["seed"] + 1000 * rank)


def make_sim(wl, state, variant):
    from miluphpc_b200 import _lib
    from miluphpc_b200.miluphpc import Miluphpc, material
    if wl["kind"] == "sph":
        # testcases/sedov: predictor-corrector, ideal gas, cubic spline,
        # Monaghan alpha = 1, beta = 2, energy integrated, density summed
        cfg = _lib.default_config(gravity=0, sph=1, integrator=1, max_time_step=wl["dt_max"], time_end=1e30,
                                  smoothing_kernel=1, integrate_energy=1, integrate_density=0, sfc=wl["sfc"],
                                  precision=wl.get("mixed_precision", 1) if variant == "mixed" else 0)
        return Miluphpc(cfg, state, materials=[material(interactions=60, alpha=1.0, beta=2.0, eos_type=9,
                                                        gamma=5.0 / 3.0)])
    if wl["kind"] == "cloud":
        # gravity (softening tied to h: eps_i = h_i / 2) + SPH (isothermal gas as
        # polytropic gamma = 1, K = c_s^2), variable h targeting 60 +- 5
        # neighbours, explicit Euler; mixed = FP32 walk + learned h, plain =
        # FP64 v2 walk (accuracy-matched theta) + plain variable-h iteration
        mixed = variant == "mixed"
        cfg = _lib.default_config(gravity=1, sph=1, integrator=0, time_step=wl["dt"], smoothing=0.0,
                                  softening_mode=1, softening_h_factor=0.5, sfc=wl["sfc"], variable_sml=1,
                                  smoothing_kernel=1, integrate_energy=0,
                                  precision=wl.get("mixed_precision", 1) if mixed else 0,
                                  theta=wl["theta"] if variant == "plain" else wl["theta_plain_matched"],
                                  theta_mixed=wl["theta_mixed"], learned_h=1 if (mixed and wl.get("learned", 1)) else 0,
                                  gravity_mac=1 if (mixed and wl.get("mac_alpha")) else 0,
                                  mac_alpha=wl.get("mac_alpha") or 0.003,
                                  mac_quad_alpha=wl.get("mac_quad_alpha", 0.0) if mixed else 0.0,
                                  sml_band_rounds=wl.get("band_rounds", 8))
        return Miluphpc(cfg, state, materials=[material(interactions=60, alpha=1.0, beta=2.0, eos_type=0,
                                                        K=state["cs2"], gamma=1.0)])
    kw = dict(gravity=1, sph=0, integrator=2, time_step=wl["dt"], smoothing=wl["eps2"], sfc=wl["sfc"],
              theta=wl["theta"], theta_mixed=wl["theta_mixed"])
    if variant == "mixed":
        kw["precision"] = wl.get("mixed_precision", 1)
        if wl.get("mac_alpha"):
            # relative opening rule from the second right-hand side on
            kw["gravity_mac"] = 1
            kw["mac_alpha"] = wl["mac_alpha"]
            kw["mac_quad_alpha"] = wl.get("mac_quad_alpha", 0.0)
    elif variant == "plain_matched":
        kw["theta"] = wl["theta_plain_matched"]
    cfg = _lib.default_config(**kw)
    return Miluphpc(cfg, state)


def force_error(sim, torch, eps2, ntarget=4096, seed=7, h_factor=0.0, h=None):
    """Relative error of the walk's accelerations against FP64 direct summation
    on a seeded sample of targets, with the walk's softening rule (eps2 plus,
    with h_factor, (h_factor h_i)^2 of the target, h_i the smoothing length
    the walk used: `h`, default the current one)."""
    from miluphpc_b200.miluphpc import direct_gravity
    n = sim.n
    rng = np.random.default_rng(seed)
    tg = np.sort(rng.choice(n, min(ntarget, n), replace=False)).astype(np.int32)
    tgt = torch.as_tensor(tg, device=sim.device)
    e2t = None
    if h_factor > 0.0:
        hh = h if h is not None else sim.t["sml"][:n]
        e2t = (h_factor * hh[tgt.long()]) ** 2
    dx, dy, dz = direct_gravity(sim.t["x"][:n], sim.t["y"][:n], sim.t["z"][:n], sim.t["mass"][:n], tgt, eps2,
                                eps2_targets=e2t)
    g = [sim.t[k][:n][tgt.long()] for k in ("g_ax", "g_ay", "g_az")]
    num = torch.sqrt((g[0] - dx) ** 2 + (g[1] - dy) ** 2 + (g[2] - dz) ** 2)
    den = torch.sqrt(dx ** 2 + dy ** 2 + dz ** 2)
    e = (num / den).cpu().numpy()
    return {"p50": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max()),
            "targets": int(len(tg))}


def cloud_energy(sim, torch):
    """Conserved quantities of the isothermal cloud: E = K + W + U with U =
    sum m c_s^2 ln rho (the isothermal internal energy, c_s^2 = K of the
    gamma = 1 polytrope; rho from the last right-hand side), W from the tree
    potential with the walk's h-tied softening, and the angular momentum."""
    d = sim.diagnostics()
    w = sim.potential()
    n = sim.n
    cs2 = float(sim.materials[0].polytropic_K)
    rho = sim.t["rho"][:n]
    u = float((sim.t["mass"][:n] * cs2 * torch.log(torch.clamp(rho, min=1e-300))).sum().item()) \
        if bool((rho > 0).all().item()) else float("nan")
    return {"E": d["kinetic"] + w + u, "L": d["angular_momentum"]}


def timed_steps(sim, step, steps, torch):
    """`steps` integration steps bracketed by CUDA events on the library's
    stream (the current torch stream), with no host synchronisation between
    them.  Returns (ms, next step)."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        sim.integrate(step)
        step += 1
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), step


def cloud_run(args, wl, variant, learned, torch, steps=None):
    """One cloud variant: the same seeded cloud, train_steps warm-up steps (the
    learned variant trains its predictor on them), one more step, then
    `steps` (default --cloud-steps) timed steps; the band and predictor
    statistics of the timed steps come from the library's device-side run
    totals, read once after them; drift of E and L over the timed steps; force
    error of an extra untimed right-hand side."""
    steps = steps or args.cloud_steps
    import ctypes
    from miluphpc_b200 import _lib
    state = plummer_state(wl, 0)
    w = dict(wl, learned=learned, band_rounds=args.band_rounds)
    sim = make_sim(w, state, variant)
    step = 0
    for _ in range(wl["train_steps"]):
        sim.integrate(step)
        step += 1
    train = None
    if variant == "mixed" and learned:
        L = _lib.load()
        l0, l1 = ctypes.c_float(), ctypes.c_float()
        t0 = time.perf_counter()
        _lib.check(L.mhpc_mlp_train(sim.ctx, 1, 1e-3, ctypes.byref(l0)), "mlp_train")
        _lib.check(L.mhpc_mlp_train(sim.ctx, wl["train_iters"], 1e-3, ctypes.byref(l1)), "mlp_train")
        train = {"plain_steps": wl["train_steps"], "iters": wl["train_iters"] + 1, "loss_first": l0.value,
                 "loss_last": l1.value, "seconds": round(time.perf_counter() - t0, 3)}
    sim.integrate(step)
    step += 1
    c0 = cloud_energy(sim, torch)
    sim.reset_run_stats()
    ms, step = timed_steps(sim, step, steps, torch)
    st = sim.stats()
    assert st["run_rhs"] == steps, (st["run_rhs"], steps)
    c1 = cloud_energy(sim, torch)
    n = sim.n
    h_walk = sim.t["sml"][:n].clone()
    sim.rhs(step)
    ferr = force_error(sim, torch, 0.0, h_factor=0.5, h=h_walk)
    l0n = float(np.linalg.norm(c0["L"]))
    out = {"ms_per_step": ms / steps, "value": n * steps / (ms / 1e3),
           "steps": steps, "force_error": ferr,
           "gravity_theta": wl["theta_mixed"] if variant == "mixed" else wl["theta_plain_matched"],
           "opening_rule": ("relative, alpha %g (geometric theta %.2f on the first RHS)" % (wl["mac_alpha"],
                                                                                        wl["theta_mixed"]))
           if variant == "mixed" else "v2 geometric (FP64)",
           "sph_pair_sums": "FP32 on hi/lo splits, FP64 accumulation" if variant == "mixed" else "FP64",
           "learned_h": bool(variant == "mixed" and learned),
           "band_rule": "reference iteration (max 5 updates, |n - 60| < 5) + %d repair rounds" % w["band_rounds"],
           "out_of_band_before_repair_rate": st["run_band_before_sum"] / st["run_band_rhs"] / n
           if st["run_band_rhs"] > 0 else None,
           "final_out_of_band_rate": st["run_out_of_band_sum"] / st["run_rhs"] / n,
           "final_out_of_band_max": int(st["run_out_of_band_max"]),
           "final_out_of_band_last_step": int(st["sml_out_of_band"]),
           "energy_rel_drift": (c1["E"] - c0["E"]) / abs(c0["E"]),
           "angular_momentum_rel_drift": float(np.linalg.norm(np.subtract(c1["L"], c0["L"]))) / l0n
           if l0n > 0 else None,
           "stages_ms_last_step": {k: round(v, 3) for k, v in st["ms_stage"].items()}}
    if variant == "mixed" and learned:
        out["first_sweep_fallback_rate"] = st["run_predictor_fallback_sum"] / st["run_rhs"] / n
        out["training"] = train
    sim.close()
    return out


def run_ours(args, wl):
    import torch
    import torch.distributed as dist
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    state = plummer_state(wl, rank)
    n = wl["n"]
    sim = make_sim(wl, state, args.variant)
    step = 0
    train_info = None
    warm = args.warmup
    # total energy K + W before the first step (gravity-only workloads; W from
    # mhpc_potential, the same tree potential at both ends)
    e_start = None
    if wl["kind"] == "gravity":
        e_start = sim.diagnostics()["kinetic"] + sim.potential()
    sim_cfg_refresh = (sim.cfg.learned_refresh_every, sim.cfg.learned_refresh_iters)
    learned_on = wl["kind"] == "cloud" and args.variant == "mixed" and wl.get("learned", 1)
    if wl["kind"] == "cloud":
        # the same start for every variant: train_steps plain steps (the
        # learned variant trains on them), then one more step
        warm = max(warm, wl["train_steps"])
    for _ in range(warm):
        sim.integrate(step)
        step += 1
    if wl["kind"] == "cloud" and not learned_on:
        sim.integrate(step)
        step += 1
    if learned_on:
        # train on the (features, converged h) pairs of the plain steps, then one
        # more step so that the first timed step starts from predictions
        import ctypes
        from miluphpc_b200 import _lib
        L = _lib.load()
        l0, l1 = ctypes.c_float(), ctypes.c_float()
        t0 = time.perf_counter()
        _lib.check(L.mhpc_mlp_train(sim.ctx, 1, 1e-3, ctypes.byref(l0)), "mlp_train")
        _lib.check(L.mhpc_mlp_train(sim.ctx, wl["train_iters"], 1e-3, ctypes.byref(l1)), "mlp_train")
        train_info = {"plain_steps": warm, "iters": wl["train_iters"] + 1, "loss_first": l0.value,
                      "loss_last": l1.value, "seconds": time.perf_counter() - t0}
        sim.integrate(step)
        step += 1
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    sph = wl["kind"] == "sph"
    # NVTX range "timed": profilers can select the timed steps' launches
    # (ncu --nvtx --nvtx-include "timed/"); the timed loop reads no statistics
    # (no host synchronisation between steps): the last timed step's counters
    # and stage events, and the library's device-side totals over the timed
    # steps, are read after it
    sim.reset_run_stats()
    step_t0 = step
    torch.cuda.nvtx.range_push("timed")
    ms, step = timed_steps(sim, step, args.steps, torch)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    value, ms_max = job_rate(ms, n, args.steps, world, dev)
    last = sim.stats()
    kern_ms = last["ms_stage"]["forces" if sph else "gravity"]
    inter = last["gravity_interactions"]
    quad = last["gravity_quad_interactions"]
    # energy drift over drift_steps steps in all (the steps after the timed
    # region run untimed)
    energy = None
    if e_start is not None:
        while step < wl.get("drift_steps", 0):
            sim.integrate(step)
            step += 1
        e_end = sim.diagnostics()["kinetic"] + sim.potential()
        energy = {"E_start": e_start, "E_end": e_end, "rel_drift": (e_end - e_start) / abs(e_start),
                  "steps": step, "potential": "tree walk, geometric rule theta_mixed, quadrupoles"}
    ferr = None
    if wl["kind"] == "gravity":
        ferr = force_error(sim, torch, wl["eps2"])
    elif wl["kind"] == "cloud":
        # explicit Euler moves the particles after its RHS: one more (untimed)
        # RHS makes the accelerations those of the current positions
        # (the walk runs before the smoothing-length update of the same RHS:
        # its softening uses the h the RHS started from)
        h_walk = sim.t["sml"][:n].clone()
        sim.rhs(step)
        ferr = force_error(sim, torch, 0.0, h_factor=0.5, h=h_walk)
    learned = None
    if wl["kind"] == "cloud":
        rr = max(last["run_rhs"], 1)
        learned = {"training": train_info, "target_band": "60 +- 5 (|n - 60| < 5)",
                   "band_repair_rounds": wl.get("band_rounds", 8), "timed_rhs": last["run_rhs"],
                   "out_of_band_before_repair_rate": last["run_band_before_sum"] / max(last["run_band_rhs"], 1) / n,
                   "fallback_rate": last["run_predictor_fallback_sum"] / rr / n,
                   "out_of_band_rate": last["run_out_of_band_sum"] / rr / n,
                   "out_of_band_max": last["run_out_of_band_max"],
                   "out_of_band_last_step": last["sml_out_of_band"]}
    # end to end through the public C ABI with host buffers (pinned)
    e2e = run_e2e(args, wl, sim, state, torch, step)
    sim.close()
    del sim
    out = None
    compare = rank == 0 and world == 1 and not args.no_compare
    vs_plain = None
    if compare and wl["kind"] == "gravity":
        vs_plain = {wl_name(args): guarded(plain_compare, args, wl, state, value, ferr, torch)}
    del state
    if compare and args.workload == "plummer16m" and args.cloud_steps > 0:
        vs_plain = vs_plain or {}
        vs_plain["cloud8m"] = guarded(cloud_compare, args, "cloud8m", args.cloud_steps, torch)
    if compare and args.workload == "plummer16m" and args.all_configs:
        vs_plain = vs_plain or {}
        # the learned-h configuration at 1M: 20 plain steps train the predictor,
        # then cloud1m_steps steps with predictor + plain fallback
        vs_plain["cloud1m"] = guarded(cloud_compare, args, "cloud1m", args.cloud1m_steps, torch)
        vs_plain["sedov2m"] = guarded(sph_compare, args, torch)
        vs_plain["plummer131k"] = guarded(small_plummer, args, torch)
    if rank == 0:
        traffic = load_traffic(args.workload, args.variant)
        if sph:
            # internal forces: the particle's own state read once (FP64: x,y,z,v,m,h,rho,p,c_s = 88 B;
            # mixed: the packed FP32 views, 56 B), the rates written (40 B) and its neighbour
            # list read (4 B per entry); neighbour gathers stay on chip (SFC order) and are
            # reported separately
            mixed = args.variant == "mixed"
            own = 56.0 if mixed else 88.0
            nb = float(last.get("mean_noi") or 0.0)
            nbytes = (own + 40.0 + 4.0 * nb) * n
            achieved = nbytes / (kern_ms / 1e3) / 1e9
            peak = hbm_peak_gbs()
            roof = {"kernel": "k_forces_f32" if mixed else "k_forces", "bound": "hbm", "achieved": round(achieved, 1),
                    "peak": peak["value"], "unit": "GB/s", "frac": round(achieved / peak["value"], 4),
                    "traffic": traffic, "peak_source": peak["source"],
                    "work_unit": "%d B state read + 40 B written + 4 B per neighbour-list entry, per particle"
                                 % own,
                    "gathered_bytes_per_launch": round(nb * n * own),
                    "kernel_ms_per_launch": round(kern_ms, 3), "mean_neighbours": nb}
        else:
            flops = inter * FLOP_MONO + quad * FLOP_QUAD
            achieved = flops / (kern_ms / 1e3) / 1e12
            peak = fp32_peak_tflops(torch)
            kname = ("k_grav_lists" if wl.get("mixed_precision", 1) == 1 else "k_grav_mixed") \
                if args.variant == "mixed" else "k_grav_v2"
            roof = {"kernel": kname, "bound": "fp32",
                    "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "TFLOP/s",
                    "frac": round(achieved / peak, 4) if peak > 0 else None, "traffic": traffic,
                    "peak_source": "FP32 FMA rate of the paired FFMA2 instruction on every SM "
                                   "(148 SMs x 128 lanes x 2 flop x the SM clock, measured by mhpc_fp32_peak)",
                    "work_unit": "%d flop per accepted monopole interaction + %d per quadrupole term"
                                 % (FLOP_MONO, FLOP_QUAD),
                    "kernel_ms_per_launch": round(kern_ms, 3), "launch": "the last timed step's walk",
                    "interactions_per_launch": inter}
        # CPU baseline: rank 0 of a single-GPU run only
        cpu = cpu_baseline(wl, args) if (not args.no_cpu_baseline and world == 1) else None
        method = {"variant": args.variant}
        if wl["kind"] == "gravity":
            method["theta"] = wl["theta_mixed"] if args.variant == "mixed" else \
                (wl["theta_plain_matched"] if args.variant == "plain_matched" else wl["theta"])
            method["opening_rule"] = ("relative: d >= l and M l^3 <= %g |a_prev| d^5, monopole cells below "
                                      "%g |a_prev| d^4 / l^2 (geometric theta %.2f on the first RHS)"
                                      % (wl["mac_alpha"], wl.get("mac_quad_alpha", 0.0), wl["theta_mixed"])) \
                if args.variant == "mixed" and wl.get("mac_alpha") and wl.get("mixed_precision", 1) == 1 \
                else "geometric"
        elif wl["kind"] == "cloud":
            method["gravity_theta"] = wl["theta_mixed"] if args.variant == "mixed" else \
                (wl["theta_plain_matched"] if args.variant == "plain_matched" else wl["theta"])
            method["learned_h"] = bool(learned_on)
        out = {
            "metric": METRIC,
            "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.variant == "mixed" else "f64",
            "data": "synthetic (seeded %s generator, no dataset)" % (
                {"sph": "Sedov lattice", "cloud": "rotating cloud", "gravity": "Plummer"}[wl["kind"]]),
            "config": workload_config(args, wl, world),
            "method": method,
            "force_error": ferr,
            "energy": energy,
            "learned_h": learned,
            "vs_plain": vs_plain,
            "stages_ms_last_step": {k: round(v, 3) for k, v in last["ms_stage"].items()},
            "tree_cells": last["cells"],
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps * launches_per_step(args.variant, wl["kind"], args.band_rounds)
            + (refresh_launches(sim_cfg_refresh, step_t0, args.steps) if learned_on else 0),
            "clocks": clk,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


METRIC = "particle-steps/s on 1 B200: mixed/learned vs plain at rel. force err <=1e-3"


def wl_name(args):
    return args.workload


def workload_config(args, wl, world):
    """The workload (identical in both arms of the bench: this library's and
    the reference's); the arm's method is reported separately."""
    n = wl["n"]
    base = {"workload": args.workload, "n_particles": n, "parallelism": "replicas" if world > 1 else "single",
            "accuracy": "p99 relative force error <= 1e-3 against FP64 direct summation (4096 seeded targets)"}
    if wl["kind"] == "sph":
        base.update({"integrator": "predictor-corrector", "kernel": "cubic spline", "h": "fixed 2.5 dx",
                     "dt_max": wl["dt_max"], "l2": "inputs larger than L2 (state %.0f MB)" % (n * 8 * 14 / 1e6)})
    elif wl["kind"] == "cloud":
        base.update({"softening": "eps_i = h_i / 2", "sph": "cubic spline, isothermal (polytropic gamma 1)",
                     "variable_h": "target 60 +- 5", "sfc": "hilbert", "integrator": "explicit euler",
                     "dt": wl["dt"], "l2": "inputs larger than L2 (state %.0f MB)" % (n * 8 * 14 / 1e6)})
    else:
        base.update({"sfc": "hilbert" if wl["sfc"] else "lebesgue", "integrator": "leapfrog", "dt": wl["dt"],
                     "eps2": wl["eps2"], "l2": "inputs larger than L2 (positions alone %.0f MB)" % (n * 24 / 1e6)})
    return base


def guarded(fn, *a, **k):
    """A comparison block: its failure is reported in the JSON line (the
    headline measurement stands on its own)."""
    try:
        return fn(*a, **k)
    except Exception as e:  # noqa: BLE001 - reported, not hidden
        return {"error": "%s: %s" % (type(e).__name__, e)}


def cloud_compare(args, name, steps, torch):
    """The cloud with the mixed walk and the learned predictor, the same
    without the predictor, and the plain FP64 path, `steps` timed steps each."""
    cw = dict(WORKLOADS[name])
    runs = {"mixed_learned": cloud_run(args, cw, "mixed", 1, torch, steps=steps),
            "mixed_no_learned": cloud_run(args, cw, "mixed", 0, torch, steps=steps),
            "plain": cloud_run(args, cw, "plain_matched", 0, torch, steps=steps)}
    runs["speedup_vs_plain"] = runs["mixed_learned"]["value"] / runs["plain"]["value"]
    runs["learned_h_gain"] = runs["mixed_learned"]["value"] / runs["mixed_no_learned"]["value"]
    runs["workload"] = "%s: rotating isothermal cloud N = %d, gravity (eps_i = h_i / 2) + SPH, variable h " \
                       "60 +- 5, explicit Euler dt %g, %d warm-up steps" % (name, cw["n"], cw["dt"],
                                                                          cw["train_steps"] + 1)
    return runs


def sph_compare(args, torch, steps=20):
    """Sedov blast (2.1M particles, SPH only, predictor-corrector): the FP32
    pair sums against the FP64 path on the same state (one right-hand side
    each: density and acceleration differences), then `steps` timed steps of
    each after one warm-up step."""
    wl = dict(WORKLOADS["sedov2m"])
    state = plummer_state(wl, 0)
    n = wl["n"]
    out = {"workload": "sedov2m: 128^3 jittered lattice, fixed h = 2.5 dx, ideal gas, predictor-corrector, "
                       "dt_max %g" % wl["dt_max"]}
    first = {}
    for variant in ("mixed", "plain"):
        sim = make_sim(wl, state, variant)
        sim.rhs(0)
        first[variant] = {k: sim.t[k][:n].clone() for k in ("rho", "ax", "ay", "az")}
        sim.close()
        sim = make_sim(wl, state, variant)
        sim.integrate(0)
        ms, _ = timed_steps(sim, 1, steps, torch)
        out[variant] = {"ms_per_step": ms / steps, "value": n * steps / (ms / 1e3), "steps": steps,
                        "sph_pair_sums": "FP32 on hi/lo splits, FP64 accumulation" if variant == "mixed"
                        else "FP64"}
        sim.close()
    a, b = first["mixed"], first["plain"]
    amax = float(torch.sqrt(b["ax"] ** 2 + b["ay"] ** 2 + b["az"] ** 2).max().item())
    out["mixed_vs_plain_first_rhs"] = {
        "density_max_rel_diff": float((a["rho"] / b["rho"] - 1).abs().max().item()),
        "acceleration_max_diff_over_max": float(max((a[k] - b[k]).abs().max().item() for k in ("ax", "ay", "az"))
                                                / amax)}
    out["speedup_vs_plain"] = out["mixed"]["value"] / out["plain"]["value"]
    return out


def small_plummer(args, torch, steps=10):
    """The reference's own single-rank case (131,072 Plummer particles,
    Lebesgue keys, theta 0.5, eps 0.01, leapfrog dt 0.025) on the plain FP64
    path with the reference's v2 semantics: time per step, force error against
    FP64 direct summation and energy drift over the steps."""
    wl = dict(WORKLOADS["plummer131k"])
    state = plummer_state(wl, 0)
    sim = make_sim(wl, state, "plain")
    e0 = sim.diagnostics()["kinetic"] + sim.potential()
    sim.integrate(0)
    sim.integrate(1)
    ms, step = timed_steps(sim, 2, steps, torch)
    st = sim.stats()
    e1 = sim.diagnostics()["kinetic"] + sim.potential()
    ferr = force_error(sim, torch, wl["eps2"])
    sim.close()
    n = wl["n"]
    return {"workload": "plummer131k: N = 131072 Plummer, Lebesgue, theta 0.5 (v2 semantics), eps2 1e-4, "
                        "leapfrog dt 0.025", "plain": {"ms_per_step": ms / steps, "value": n * steps / (ms / 1e3),
                                                       "steps": steps, "force_error": ferr,
                                                       "energy_rel_drift": (e1 - e0) / abs(e0),
                                                       "energy_steps": step,
                                                       "stages_ms_last_step": {k: round(v, 3) for k, v in
                                                                               st["ms_stage"].items()}}}


def plain_compare(args, wl, state, mixed_value, mixed_ferr, torch):
    """The plain FP64 walk (computeForces_v2 semantics) on the same workload
    at the opening parameter whose p99 force error matches the mixed run's."""
    sim = make_sim(wl, state, "plain_matched")
    step = 0
    for _ in range(max(1, args.plain_warmup)):
        sim.integrate(step)
        step += 1
    ms, step = timed_steps(sim, step, args.plain_steps, torch)
    ferr = force_error(sim, torch, wl["eps2"])
    sim.close()
    value = wl["n"] * args.plain_steps / (ms / 1e3)
    return {"mixed": {"value": mixed_value, "force_error_p99": mixed_ferr["p99"] if mixed_ferr else None},
            "plain": {"value": value, "ms_per_step": ms / args.plain_steps, "steps": args.plain_steps,
                      "theta": wl["theta_plain_matched"], "force_error": ferr, "walk": "FP64 v2 (warp vote)"},
            "speedup_vs_plain": mixed_value / value,
            "p99_ratio_plain_over_mixed": (ferr["p99"] / mixed_ferr["p99"]) if mixed_ferr else None}


def hbm_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return {"value": float(json.load(open(p))["hbm_gbs"]), "source": "MEASURED_PEAKS.json hbm_gbs (measured)"}
    except Exception:
        return {"value": 6650.0, "source": "fallback 6.65 TB/s"}


def launches_per_step(variant, kind="gravity", band_rounds=8):
    """This library's kernel launches in one timed step (counted from the
    launch sequence; the ncu launch lists in profiles/ show the same)."""
    # every RHS: bbox, bbox_finish, keys, hist, hist_scan, 8 onesweep (13), gather (1),
    # tree: lcp, count, 4 scan, copy_total, zero_cells, nodes (9), upward pass (1)
    tree = 13 + 1 + 9 + 1
    mixed = variant == "mixed"
    if kind == "sph":
        # frnn, (mixed: position pack), density+EOS, forces; noi export on the
        # first RHS only; predictor-corrector: 3 step-size kernels, predictor, corrector
        # (+1: the status fold at the start of every SPH right-hand side)
        rhs = 1 + tree + 1 + (1 if mixed else 0) + 2
        return (rhs + 1) + rhs + 3 + 2
    grav = tree + 1  # + the walk
    if kind == "cloud":
        # variable h on lists: copy of h, largest-h bounds (one upward pass), the
        # list walk of the starting h, the first sweep's list (flags, 4 scan,
        # compact), 7 sweeps x (update, event reset, events, marks, filter, appends,
        # commit, gated re-walk), the next list of each later sweep (6), record after
        # the first sweep, final list + record, sort of the appended lists, list
        # statistics, scatter of h; band repair: 2 copies,
        # rounds x (flags, 4 scan, compact, select, events, remove, compact, add,
        # commit), sort of the appended lists, scatter of h; (mixed: position pack)
        # density, forces, noi export, band statistics; learned h: apply, collect,
        # features; explicit Euler update
        vh = 1 + 1 + 1 + 6 + 7 * 8 + 6 + 1 + 2 + 1 + 1 + 1
        band = (2 + 12 * band_rounds + 1 + 1) if band_rounds > 0 else 0
        sphk = band + (1 if mixed else 0) + 4
        learned = 3 if mixed else 0
        return 1 + grav + vh + sphk + learned + 1  # status fold, ..., explicit Euler
    return grav + 2  # leapfrog updateX, updateV


def refresh_launches(every_iters, step0, steps):
    """Launches of the learned predictor's refreshes inside the timed steps:
    k_train, Adam and the BF16 mirror per Adam step, at every right-hand side
    whose count since the context's creation is a multiple of `every` (one RHS
    per explicit Euler step, counted from 1)."""
    every, iters = every_iters
    if every <= 0:
        return 0
    return 3 * iters * sum(1 for r in range(step0 + 1, step0 + steps + 1) if r % every == 0)


def run_e2e(args, wl, sim, state, torch, step0):
    """Same steps through mhpc_integrate_host_async (+ mhpc_host_wait): host (pinned) state copied in
    and the new state + accelerations copied out every step."""
    import ctypes
    from miluphpc_b200 import _lib
    n = sim.n
    if wl["kind"] in ("sph", "cloud"):
        fields_in = ["x", "y", "z", "mass", "vx", "vy", "vz", "sml", "e", "rho", "p", "cs", "ax", "ay", "az",
                     "g_ax", "g_ay", "g_az"]
        n_in, n_out = 12, 14 if wl["kind"] == "sph" else 17
    else:
        fields_in = ["x", "y", "z", "mass", "vx", "vy", "vz", "g_ax", "g_ay", "g_az"]
        n_in, n_out = 10, 9
    host = {}
    for f in fields_in:
        host[f] = torch.empty(n, dtype=torch.float64, pin_memory=True)
        host[f].copy_(sim.t[f][:n].cpu())
    hp = _lib.Particles()
    hp.n = n
    hp.num_nodes = n
    for f in fields_in:
        setattr(hp, f, ctypes.cast(ctypes.c_void_p(host[f].data_ptr()), _lib.P_d))
    L = _lib.load()
    dt = ctypes.c_double()
    steps = max(2, args.steps)
    # one untimed call allocates the context's device mirrors; the timed steps
    # (as many as the device-resident measurement) overlap each step's copy-in
    # with the previous step's compute and copy-out (mhpc_integrate_host_async),
    # the last wait inside the timed region
    _lib.check(L.mhpc_integrate_host(sim.ctx, ctypes.byref(hp), step0, ctypes.byref(dt)), "integrate_host")
    t0 = time.perf_counter()
    for k in range(steps):
        _lib.check(L.mhpc_integrate_host_async(sim.ctx, ctypes.byref(hp), step0 + 1 + k, ctypes.byref(dt)),
                   "integrate_host_async")
    _lib.check(L.mhpc_host_wait(sim.ctx), "host_wait")
    el = time.perf_counter() - t0
    h2d = n_in * 8 * n
    d2h = n_out * 8 * n
    return {"value": n * steps / el, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps}


def load_traffic(workload, variant):
    """DRAM bytes (read + write) per launch of the dominant kernel, from the
    `traffic <workload>/<variant> <bytes>` lines of the committed ncu
    summaries under profiles/ (None when no capture covers the workload)."""
    import glob
    key = "%s/%s" % (workload, variant)
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for line in open(path):
            f = line.split()
            if len(f) == 3 and f[0] == "traffic" and f[1] == key:
                return float(f[2])
    return None


def cpu_baseline(wl, args, sample_groups=None):
    """The reference algorithm (FP64 v2 walk at the accuracy-matched theta,
    with keys, sort, tree and COM) restated by the oracle, timed on the host
    cores: full keys/sort/tree/COM on all particles, the walk on a sample of
    warp groups, scaled to the full workload."""
    from oracle import oracle as O
    from miluphpc_b200 import ics
    n = wl["n"]
    if wl["kind"] == "cloud":
        return None
    if wl["kind"] == "sph":
        # neighbours, density, EOS and forces of one RHS on all particles;
        # a predictor-corrector step runs two of them
        S = ics.sedov(nside=wl["nside"], seed=wl["seed"])
        t0 = time.perf_counter()
        off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
        rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr)
        p, cs = O.eos(9, np.array([0.0, 5.0 / 3.0, 0, 0, 0]), rho, S["e"], np.zeros(n))
        O.forces(S["x"], S["y"], S["z"], S["vx"], S["vy"], S["vz"], S["mass"], S["sml"], rho, p, cs, off, nbr,
                 1.0, 2.0)
        t1 = time.perf_counter()
        return {"value": n / (2 * (t1 - t0)), "unit": "particle-steps/s", "cores": O.num_threads(), "kind": "port",
                "sample": "one full SPH RHS (neighbours, density, EOS, forces) on all %d particles (%.1f s), x2 "
                          "for the two RHS of a predictor-corrector step" % (n, t1 - t0),
                "seconds": t1 - t0}
    P = ics.plummer(n, seed=wl["seed"])
    theta = wl["theta_plain_matched"]
    t0 = time.perf_counter()
    bb = O.bbox(P["x"], P["y"], P["z"])
    k = O.keys(P["x"], P["y"], P["z"], bb, wl["sfc"])
    _, perm = O.sort(k)
    t1 = time.perf_counter()
    T = O.Tree(P["x"], P["y"], P["z"], P["mass"], bb)
    t2b = time.perf_counter()
    ngroups = (n + 31) // 32
    radius = 0.5 * (bb[1] - bb[0])
    stride = max(1, ngroups // (sample_groups or args.cpu_sample_groups))
    t2 = time.perf_counter()
    O.gravity_v2_sample(T, perm, radius, theta, wl["eps2"], stride)
    t3 = time.perf_counter()
    # grow the walk sample to about 5 s of host time so that the scaled figure
    # is not dominated by noise
    if t3 - t2 < 1.0 and stride > 1:
        stride = max(1, int(stride * (t3 - t2) / 5.0))
        t2 = time.perf_counter()
        O.gravity_v2_sample(T, perm, radius, theta, wl["eps2"], stride)
        t3 = time.perf_counter()
    sampled = len(range(0, ngroups, stride))
    walk_full = (t3 - t2) * ngroups / sampled
    total = (t1 - t0) + (t2b - t1) + walk_full
    return {"value": n / total, "unit": "particle-steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": "keys+sort+tree+COM on all %d particles (%.2f s), v2 walk (theta %.2f) on %d of %d warp "
                      "groups (every %d-th, %.2f s) scaled x%.1f" % (n, (t1 - t0) + (t2b - t1), theta, sampled,
                                                                 ngroups, stride, t3 - t2, ngroups / sampled),
            "seconds": (t1 - t0) + (t2b - t1) + (t3 - t2)}


def run_reference(args, wl):
    rank, world, _ = rank_info()
    if rank != 0:
        return None
    per_step = []
    cb = None
    # one untimed sample stands for the warm-up steps (each sample is ~10 s of
    # CPU work; W of them would not fit the run's few minutes)
    if args.warmup > 0:
        cpu_baseline(wl, args, sample_groups=args.cpu_sample_groups)
    for s in range(max(1, args.steps)):
        cb = cpu_baseline(wl, args, sample_groups=args.cpu_sample_groups)
        per_step.append(cb["value"])
    value = float(np.median(per_step))
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wl["n"] / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Plummer sampler, no dataset)",
        "config": workload_config(args, wl, world),
        "method": {"variant": "reference algorithm (computeForces_v2 semantics, FP64) restated by the CPU oracle",
                   "theta": wl["theta_plain_matched"], "opening_rule": "geometric"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plummer16m", choices=sorted(WORKLOADS))
    ap.add_argument("--variant", default="mixed", choices=["mixed", "plain", "plain_matched"])
    ap.add_argument("--cpu-sample-groups", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the plain FP64 comparison runs (single-GPU runs only make them)")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed steps of the plain FP64 comparison")
    ap.add_argument("--plain-warmup", type=int, default=1)
    ap.add_argument("--cloud-steps", type=int, default=100,
                    help="timed steps of each cloud8m comparison run (0: no cloud comparison)")
    ap.add_argument("--cloud1m-steps", type=int, default=200, help="timed steps of each cloud1m comparison run")
    ap.add_argument("--no-all-configs", dest="all_configs", action="store_false",
                    help="skip the cloud1m, sedov2m and plummer131k comparison blocks")
    ap.add_argument("--theta-mixed", type=float, default=None, help="override the mixed walk's opening parameter")
    ap.add_argument("--theta-plain", type=float, default=None,
                    help="override the accuracy-matched opening parameter of the plain FP64 walk")
    ap.add_argument("--mac-alpha", type=float, default=None,
                    help="relative opening rule of the list walk (0: geometric rule only)")
    ap.add_argument("--mac-quad-alpha", type=float, default=None,
                    help="relative rule: cells with a small quadrupole term enter as monopoles (0: never)")
    ap.add_argument("--learned", type=int, default=1, help="cloud workloads, mixed variant: learned-h predictor on/off")
    ap.add_argument("--band-rounds", type=int, default=8,
                    help="cloud workloads: neighbour-band repair rounds after the variable-h iteration (0: none)")
    ap.add_argument("--mixed-walk", default="lists", choices=["lists", "vote"],
                    help="mixed walk: interaction lists (precision 1) or per-lane vote (precision 2)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.theta_mixed is not None:
        wl["theta_mixed"] = args.theta_mixed
    if args.mac_alpha is not None:
        wl["mac_alpha"] = args.mac_alpha
    if args.mac_quad_alpha is not None:
        wl["mac_quad_alpha"] = args.mac_quad_alpha
    if args.theta_plain is not None:
        wl["theta_plain_matched"] = args.theta_plain
    wl["mixed_precision"] = 1 if args.mixed_walk == "lists" else 2
    wl["learned"] = args.learned
    wl["band_rounds"] = args.band_rounds
    if args.impl == "reference":
        out = run_reference(args, wl)
    else:
        out = run_ours(args, wl)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
