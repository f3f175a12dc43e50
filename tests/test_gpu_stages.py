"""Parity of the per-stage exports, the integrator update kernels, the
diagnostics, the non-cubic smoothing kernels, the other equations of state,
a combined gravity + SPH + variable-h right-hand side, and the neighbour-band
repair, all through the C ABI against the FP64 oracle.

Bars: integrator updates bit-identical to the oracle (both round every
product and sum separately, like the reference's -fmad=false build); the
per-stage sequence bit-identical to mhpc_rhs; FP64 SPH sums within 1e-12
(density, p, c_s) and 1e-10 of the largest magnitude (rates); FP32 pair sums
within 2e-6 (density) and 2e-5 of the largest magnitude (rates); the band
repair's h bit-identical to the oracle's rule started from the same h, and
every list equal to the brute-force set of the repaired h.
"""
import ctypes

import numpy as np
import pytest
import torch

from miluphpc_b200 import _lib, ics
from miluphpc_b200.miluphpc import Miluphpc, material
from oracle import oracle as O
from tests.helpers import gravity_cfg, rel_err, sph_cfg

pytestmark = pytest.mark.gpu


def L():
    return _lib.load()


def _sedov_state(nside, seed=5, vel=0.05):
    S = ics.sedov(nside=nside, seed=seed)
    rng = np.random.default_rng(seed)
    n = len(S["x"])
    for k in ("vx", "vy", "vz"):
        S[k] = rng.normal(0.0, vel, n)
    S["p"] = np.zeros(n)
    S["cs"] = np.zeros(n)
    return S


def _cloud_state(n, seed=4, spread=(0.85, 1.15), vel_noise=0.05):
    """Rotating cloud with h spread around the mean-density value and random
    velocities added to the solid-body rotation (whose divergence is zero, so
    that d rho / dt would be rounding noise alone)."""
    C = ics.rotating_cloud(n, seed=seed)
    S = dict(C)
    m = len(S["x"])
    S["sml"] = C["sml"] * np.random.default_rng(2).uniform(spread[0], spread[1], m)
    for k in ("vx", "vy", "vz"):
        S[k] = S[k] + np.random.default_rng(5).normal(0.0, vel_noise, m)
    S["p"] = np.zeros(m)
    S["cs"] = np.zeros(m)
    return S, C


def _random_state(n, seed, fields):
    rng = np.random.default_rng(seed)
    st = {}
    for f in fields:
        st[f] = rng.normal(0.0, 1.0, n)
    for f in ("sml", "rho", "e", "mass"):
        if f in st:
            st[f] = np.abs(st[f]) + 0.1
    return st


# ------------------------------------------------------------- integrators
def test_euler_update_bit_exact(cuda):
    """ExplicitEulerNS::Kernel::update through mhpc_integrate_euler against the
    oracle's restatement, every switch on, with the e >= 1e-50 floor hit."""
    n = 10_000
    fields = ["x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay", "g_az", "rho", "drhodt",
              "e", "dedt", "sml", "dsmldt", "mass", "p", "cs"]
    st = _random_state(n, 3, fields)
    st["dedt"][:100] = -1e6  # e + dt dedt < 0: floored at 1e-50
    cfg = sph_cfg(gravity=1, integrate_density=1, integrate_energy=1, integrate_sml=1)
    sim = Miluphpc(cfg, st)
    dt = 3.7e-3
    _lib.check(L().mhpc_integrate_euler(sim.ctx, ctypes.byref(sim.soa), dt), "integrate_euler")
    torch.cuda.synchronize()
    ref = O.euler(st, dt, gravity=True, sph=True, integrate_density=True, integrate_energy=True,
                  integrate_sml=True)
    for f in ("x", "y", "z", "vx", "vy", "vz", "rho", "e", "sml"):
        assert np.array_equal(sim.numpy(f), ref[f]), f
    assert (sim.numpy("e")[:100] == 1e-50).all()
    sim.close()
    # gravity only: the SPH accelerations are not read
    cfg = gravity_cfg(integrator=0)
    st2 = _random_state(n, 4, ["x", "y", "z", "vx", "vy", "vz", "g_ax", "g_ay", "g_az", "mass"])
    sim = Miluphpc(cfg, st2)
    sim.t["ax"].fill_(1e300)
    _lib.check(L().mhpc_integrate_euler(sim.ctx, ctypes.byref(sim.soa), dt), "integrate_euler")
    torch.cuda.synchronize()
    ref = O.euler(st2, dt, gravity=True, sph=False)
    for f in ("x", "vx", "vz"):
        assert np.array_equal(sim.numpy(f), ref[f]), f
    sim.close()


def test_leapfrog_updates_bit_exact(cuda):
    n = 10_000
    fields = ["x", "y", "z", "vx", "vy", "vz", "g_ax", "g_ay", "g_az", "g_ax_old", "g_ay_old", "g_az_old",
              "mass"]
    st = _random_state(n, 7, fields)
    sim = Miluphpc(gravity_cfg(), st)
    dt = 0.025
    _lib.check(L().mhpc_integrate_leapfrog(sim.ctx, ctypes.byref(sim.soa), dt, 0), "leapfrog x")
    ref = {k: np.array(v, copy=True) for k, v in st.items()}
    p = O._p
    O.lib().orc_leapfrog_x(n, dt, *[p(ref[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "g_ax", "g_ay", "g_az",
                                                          "g_ax_old", "g_ay_old", "g_az_old")])
    torch.cuda.synchronize()
    for f in ("x", "y", "z", "g_ax_old"):
        assert np.array_equal(sim.numpy(f), ref[f]), f
    # new accelerations, then the kick
    g = np.random.default_rng(8).normal(0.0, 1.0, (3, n))
    for k, a in zip(("g_ax", "g_ay", "g_az"), g):
        sim.t[k][:n] = torch.as_tensor(a, device=cuda)
        ref[k] = a.copy()
    _lib.check(L().mhpc_integrate_leapfrog(sim.ctx, ctypes.byref(sim.soa), dt, 1), "leapfrog v")
    O.lib().orc_leapfrog_v(n, dt, *[p(ref[k]) for k in ("vx", "vy", "vz", "g_ax", "g_ay", "g_az", "g_ax_old",
                                                          "g_ay_old", "g_az_old")])
    torch.cuda.synchronize()
    for f in ("vx", "vy", "vz"):
        assert np.array_equal(sim.numpy(f), ref[f]), f
    with pytest.raises(_lib.MhpcError):
        _lib.check(L().mhpc_integrate_leapfrog(sim.ctx, ctypes.byref(sim.soa), dt, 2), "bad half")
    sim.close()


def test_pc_step_size_predictor_corrector(cuda):
    """setTimeStep, predictor and corrector of the predictor-corrector Euler
    through their exports: the update kernels bit-identical to a numpy
    restatement (elementwise IEEE double, no contraction), the step size
    equal to the oracle's formula."""
    n = 8192
    fields = ["x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay", "g_az", "rho", "drhodt",
              "e", "dedt", "sml", "dsmldt", "mass", "p", "cs"]
    st = _random_state(n, 11, fields)
    st["cs"] = np.abs(st["cs"]) + 0.5
    cfg = sph_cfg(gravity=1, integrator=1, integrate_density=1, integrate_energy=1, integrate_sml=1,
                  max_time_step=1.0)
    mat = material(interactions=60, alpha=1.0, beta=2.0, eos_type=9)
    sim = Miluphpc(cfg, st, materials=[mat])
    q = Miluphpc(cfg, _random_state(n, 12, fields), materials=[mat])  # predicted state (IntegratedParticles)
    dt_dev = torch.zeros(1, dtype=torch.float64, device=cuda)
    _lib.check(L().mhpc_integrate_pc_step_size(sim.ctx, ctypes.byref(sim.soa), 1e30,
                                               ctypes.c_void_p(dt_dev.data_ptr())), "step size")
    torch.cuda.synchronize()
    a = np.sqrt((st["ax"] + st["g_ax"]) ** 2 + (st["ay"] + st["g_ay"]) ** 2 + (st["az"] + st["g_az"]) ** 2)
    forces = np.min(np.sqrt(st["sml"] / a))
    courant = np.min(st["sml"] / st["cs"])
    visc = np.min(0.4 * st["sml"] / (st["cs"] + 1.2 * (1.0 * st["cs"])))
    nz = st["drhodt"] != 0
    dtrho = np.min(0.1 * (np.abs(st["rho"][nz]) + 0.001) / np.abs(st["drhodt"][nz]))
    dt_ref = min(0.4 * courant, 0.2 * forces, visc, dtrho)
    dt = float(dt_dev.item())
    # the reference's v_max combine (minimum of block maxima) may also cap it
    assert dt <= dt_ref * (1 + 1e-14) and dt > 0
    _lib.check(L().mhpc_integrate_pc_predictor(sim.ctx, ctypes.byref(sim.soa), ctypes.byref(q.soa),
                                               ctypes.c_void_p(dt_dev.data_ptr())), "predictor")
    torch.cuda.synchronize()
    P = {k: st[k] for k in fields}
    Q = {k: q.numpy(k) for k in fields}
    for c, v, g, s in (("x", "vx", "g_ax", "ax"), ("y", "vy", "g_ay", "ay"), ("z", "vz", "g_az", "az")):
        assert np.array_equal(Q[c], P[c] + dt * P[v]), c
        assert np.array_equal(Q[v], P[v] + dt * (P[s] + P[g])), v
    assert np.array_equal(Q["rho"], P["rho"] + dt * P["drhodt"])
    assert np.array_equal(Q["e"], np.maximum(P["e"] + dt * P["dedt"], 1e-6))
    # rates of the predicted state (a right-hand side on q would write them)
    R = _random_state(n, 13, ["ax", "ay", "az", "drhodt", "dedt", "dsmldt"])
    for k, v in R.items():
        q.t[k][:n] = torch.as_tensor(v, device=cuda)
        Q[k] = v
    _lib.check(L().mhpc_integrate_pc_corrector(sim.ctx, ctypes.byref(sim.soa), ctypes.byref(q.soa),
                                               ctypes.c_void_p(dt_dev.data_ptr())), "corrector")
    torch.cuda.synchronize()
    h = 0.5 * dt
    for c, v, a, g in (("x", "vx", "ax", "g_ax"), ("y", "vy", "ay", "g_ay"), ("z", "vz", "az", "g_az")):
        assert np.array_equal(sim.numpy(c), P[c] + h * (Q[v] + P[v])), c
        assert np.array_equal(sim.numpy(v), P[v] + h * ((Q[a] + P[a]) + 2.0 * P[g])), v
        assert np.array_equal(sim.numpy(a), 0.5 * (Q[a] + P[a]) + P[g]), a
    assert np.array_equal(sim.numpy("rho"), P["rho"] + h * (Q["drhodt"] + P["drhodt"]))
    assert np.array_equal(sim.numpy("e"), np.maximum(P["e"] + h * (Q["dedt"] + P["dedt"]), 1e-6))
    assert np.array_equal(sim.numpy("sml"), P["sml"] + h * (Q["dsmldt"] + P["dsmldt"]))
    sim.close()
    q.close()


def test_diagnostics_match_numpy(cuda):
    """Energies, linear and angular momentum and centre of mass
    (Miluphpc::totalEnergy / angularMomentum, src/miluphpc.cpp:577-677)."""
    S, _ = _cloud_state(30_000)
    S["e"] = np.random.default_rng(3).uniform(0.1, 1.0, len(S["x"]))
    sim = Miluphpc(sph_cfg(gravity=1), S, materials=[material(eos_type=0, K=0.1, gamma=1.0)])
    d = sim.diagnostics()
    m, x, y, z = S["mass"], S["x"], S["y"], S["z"]
    vx, vy, vz = S["vx"], S["vy"], S["vz"]
    np.testing.assert_allclose(d["kinetic"], 0.5 * np.sum(m * (vx ** 2 + vy ** 2 + vz ** 2)), rtol=1e-12)
    np.testing.assert_allclose(d["internal"], np.sum(m * S["e"]), rtol=1e-12)
    np.testing.assert_allclose(d["momentum"], [np.sum(m * vx), np.sum(m * vy), np.sum(m * vz)], rtol=1e-9,
                               atol=1e-15)
    L_ref = [np.sum(m * (y * vz - z * vy)), np.sum(m * (z * vx - x * vz)), np.sum(m * (x * vy - y * vx))]
    np.testing.assert_allclose(d["angular_momentum"], L_ref, rtol=1e-12, atol=1e-15)
    M = np.sum(m)
    np.testing.assert_allclose(d["com"], [np.sum(m * x) / M, np.sum(m * y) / M, np.sum(m * z) / M], rtol=1e-9,
                               atol=1e-15)
    sim.close()


# ------------------------------------------------- kernels and EOS types
@pytest.mark.parametrize("kernel", [0, 2, 3, 4])
@pytest.mark.parametrize("precision", [0, 1])
def test_smoothing_kernels(kernel, precision, cuda):
    """Spiky and Wendland C2/C4/C6 (SmoothingKernel, src/sph/kernel.cu:14-183)
    in the density and force sums against the oracle's restatement."""
    S = _sedov_state(20)
    n = len(S["x"])
    cfg = sph_cfg(smoothing_kernel=kernel, precision=precision)
    mat = material(interactions=60, alpha=1.0, beta=2.0, eos_type=9, gamma=5.0 / 3.0)
    sim = Miluphpc(cfg, S, materials=[mat])
    sim.rhs(0)
    sim.rhs(1)
    off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr, kernel=kernel)
    par = np.array([0.0, 5.0 / 3.0, 0.0, 0.0, 0.0])
    p0, _ = O.eos(9, par, O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr, kernel=kernel),
                  S["e"], np.zeros(n))
    p, cs = O.eos(9, par, rho, S["e"], p0)
    ax, ay, az, drho, de, _ = O.forces(S["x"], S["y"], S["z"], S["vx"], S["vy"], S["vz"], S["mass"], S["sml"],
                                       rho, p, cs, off, nbr, 1.0, 2.0, kernel=kernel)
    rtol_rho, frac = (1e-12, 1e-10) if precision == 0 else (2e-6, 2e-5)
    np.testing.assert_allclose(sim.numpy("rho"), rho, rtol=rtol_rho)
    scale = np.abs(np.stack([ax, ay, az])).max()
    for got, ref in ((sim.numpy("ax"), ax), (sim.numpy("ay"), ay), (sim.numpy("az"), az)):
        np.testing.assert_allclose(got, ref, rtol=0, atol=frac * scale)
    np.testing.assert_allclose(sim.numpy("drhodt"), drho, rtol=0, atol=frac * np.abs(drho).max())
    np.testing.assert_allclose(sim.numpy("dedt"), de, rtol=0, atol=frac * np.abs(de).max())
    sim.close()


@pytest.mark.parametrize("eos", [1, 3, 12])
def test_equations_of_state(eos, cuda):
    """Murnaghan (1), isothermal H2 (3) and locally isothermal (12)
    pressures and sound speeds (src/sph/pressure.cu:5-44, soundspeed.cu:4-97),
    and the forces that follow, against the oracle."""
    S = _sedov_state(16)
    n = len(S["x"])
    S["cs"] = np.full(n, 0.3)
    m = material(interactions=60, alpha=1.0, beta=2.0, eos_type=eos)
    m.rho_0 = 0.9
    m.bulk_modulus = 2.5
    m.n = 7.0
    sim = Miluphpc(sph_cfg(), S, materials=[m])
    sim.rhs(0)
    off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr)
    p, cs = O.eos(eos, np.array([0.0, 5.0 / 3.0, 0.9, 2.5, 7.0]), rho, S["e"], np.zeros(n))
    if eos == 12:
        assert (cs == 0).all()
    np.testing.assert_allclose(sim.numpy("p"), p, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(sim.numpy("cs"), cs, rtol=1e-15, atol=0)
    ax, ay, az, drho, de, _ = O.forces(S["x"], S["y"], S["z"], S["vx"], S["vy"], S["vz"], S["mass"], S["sml"],
                                       rho, p, cs, off, nbr, 1.0, 2.0)
    scale = np.abs(np.stack([ax, ay, az])).max()
    for got, ref in ((sim.numpy("ax"), ax), (sim.numpy("ay"), ay), (sim.numpy("az"), az)):
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * scale)
    sim.close()


# ------------------------------------------- combined right-hand side
def _combined_cfg(**kw):
    base = dict(gravity=1, sph=1, integrator=0, time_step=1e-3, sfc=0, theta=0.5, smoothing=1e-4,
                variable_sml=1, integrate_energy=0, smoothing_kernel=1)
    base.update(kw)
    return _lib.default_config(**base)


def test_combined_gravity_sph_variable_h(cuda):
    """One right-hand side with self-gravity (v2 walk), the variable-h
    iteration, density, polytropic EOS and forces on a 20 K cloud, then the
    explicit Euler update of mhpc_integrate, against the oracle."""
    S, C = _cloud_state(20_000)
    n = len(S["x"])
    mat = material(interactions=60, alpha=1.0, beta=2.0, eos_type=0, K=C["cs2"], gamma=1.0)
    sim = Miluphpc(_combined_cfg(), S, materials=[mat], want_nnl=True)
    sim.rhs(0)
    # gravity: the oracle's v2 emulation on the same tree
    bb = O.bbox(S["x"], S["y"], S["z"])
    _, perm = O.sort(O.keys(S["x"], S["y"], S["z"], bb, 0))
    T = O.Tree(S["x"], S["y"], S["z"], S["mass"], bb)
    gx, gy, gz = O.gravity_v2(T, perm, 0.5 * (bb[1] - bb[0]), 0.5, 1e-4)
    e = rel_err(sim.numpy("g_ax"), sim.numpy("g_ay"), sim.numpy("g_az"), gx, gy, gz)
    assert e.max() < 1e-9, e.max()
    # variable h: the oracle's Jacobi iteration
    h_gpu = sim.numpy("sml")
    h_orc, _, _ = O.variable_h(S["x"], S["y"], S["z"], S["sml"], 60, tol=5, max_nb=180, max_iter=5)
    assert (np.abs(h_gpu - h_orc) <= 1e-12 * h_orc).mean() > 0.999
    # lists, density, EOS and forces on the GPU's h
    off, nbr = O.frnn(S["x"], S["y"], S["z"], h_gpu)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, np.diff(off))
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, 180)
    for i in range(0, n, 13):
        assert np.array_equal(np.sort(nnl[i, :noi[i]]), nbr[off[i]:off[i + 1]])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], h_gpu, off, nbr, avg_h=True)
    np.testing.assert_allclose(sim.numpy("rho"), rho, rtol=1e-12)
    p, cs = O.eos(0, np.array([float(C["cs2"]), 1.0, 0, 0, 0]), rho, S["e"], np.zeros(n))
    np.testing.assert_allclose(sim.numpy("p"), p, rtol=1e-12)
    np.testing.assert_allclose(sim.numpy("cs"), cs, rtol=1e-12)
    ax, ay, az, drho, _, _ = O.forces(S["x"], S["y"], S["z"], S["vx"], S["vy"], S["vz"], S["mass"], h_gpu, rho,
                                      p, cs, off, nbr, 1.0, 2.0, avg_h=True, integrate_energy=False)
    scale = np.abs(np.stack([ax, ay, az])).max()
    for got, ref in ((sim.numpy("ax"), ax), (sim.numpy("ay"), ay), (sim.numpy("az"), az)):
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(sim.numpy("drhodt"), drho, rtol=0, atol=1e-10 * np.abs(drho).max())
    sim.close()
    # mhpc_integrate (explicit Euler): the update applied to its own RHS output
    sim = Miluphpc(_combined_cfg(), S, materials=[mat])
    sim.rhs(0)
    st = {k: sim.numpy(k).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay",
                                           "g_az", "sml")}
    sim2 = Miluphpc(_combined_cfg(), S, materials=[mat])
    sim2.integrate(0)
    ref = O.euler(st, 1e-3, gravity=True, sph=True)
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(sim2.numpy(f), ref[f]), f
    sim.close()
    sim2.close()


def test_stage_exports_equal_rhs(cuda):
    """mhpc_tree_build, mhpc_com, mhpc_gravity, mhpc_frnn, mhpc_density_eos and
    mhpc_forces in sequence give mhpc_rhs's outputs bit for bit; stages out of
    order are refused."""
    S, C = _cloud_state(20_000, seed=6)
    mat = material(interactions=60, alpha=1.0, beta=2.0, eos_type=0, K=C["cs2"], gamma=1.0)
    cfg = _combined_cfg(precision=1, theta_mixed=0.3)
    a = Miluphpc(cfg, S, materials=[mat])
    a.rhs(0)
    b = Miluphpc(cfg, S, materials=[mat])
    lib = L()
    sp = ctypes.byref(b.soa)
    with pytest.raises(_lib.MhpcError):
        _lib.check(lib.mhpc_density_eos(b.ctx, sp), "density before frnn")
    with pytest.raises(_lib.MhpcError):
        _lib.check(lib.mhpc_gravity(b.ctx, sp, -1), "gravity before tree")
    _lib.check(lib.mhpc_tree_build(b.ctx, sp), "tree_build")
    _lib.check(lib.mhpc_com(b.ctx, sp), "com")
    _lib.check(lib.mhpc_gravity(b.ctx, sp, -1), "gravity")
    _lib.check(lib.mhpc_frnn(b.ctx, sp, 1, 0), "frnn")
    _lib.check(lib.mhpc_density_eos(b.ctx, sp), "density_eos")
    _lib.check(lib.mhpc_forces(b.ctx, sp), "forces")
    _lib.check(lib.mhpc_ctx_status(b.ctx), "status")
    for f in ("g_ax", "g_ay", "g_az", "sml", "rho", "p", "cs", "ax", "ay", "az", "drhodt"):
        assert np.array_equal(a.numpy(f), b.numpy(f)), f
    # the plain walk on the same context (its own precision argument)
    _lib.check(lib.mhpc_gravity(b.ctx, sp, 0), "gravity plain")
    _lib.check(lib.mhpc_ctx_status(b.ctx), "status")
    assert np.isfinite(b.numpy("g_ax")).all()
    a.close()
    b.close()


# ------------------------------------------------- neighbour-band repair
def test_band_repair_matches_oracle(cuda):
    """The band repair (sml_band_rounds) from the h the variable-h iteration
    left: the final h equal to the oracle's rule on the same start, every
    neighbour list equal to the brute-force set of the final h, and the only
    particles left outside 60 +- 5 those below the band whose h reached the
    repair's cap (twice the h of the first round): their neighbours' h do not
    reach them, so their own h alone cannot add pairs."""
    S, C = _cloud_state(20_000)
    n = len(S["x"])
    mat = material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)
    sim0 = Miluphpc(sph_cfg(variable_sml=1, integrate_energy=0), S, materials=[mat])
    sim0.rhs(0)
    h_jacobi = sim0.numpy("sml")
    before = int(np.sum(np.abs(sim0.numpy("noi") - 60) >= 5))
    sim0.close()
    sim = Miluphpc(sph_cfg(variable_sml=1, integrate_energy=0, sml_band_rounds=8), S, materials=[mat],
                   want_nnl=True)
    sim.rhs(0)
    st = sim.stats()
    assert st["sml_band_before"] == before and before > 100 and st["sml_band_skipped"] == 0
    h_gpu = sim.numpy("sml")
    h_orc, b_orc = O.band_fixup(S["x"], S["y"], S["z"], h_jacobi, 60, tol=5, rounds=8)
    assert b_orc == before
    assert np.array_equal(h_gpu, h_orc), np.sum(h_gpu != h_orc)
    off, nbr = O.frnn(S["x"], S["y"], S["z"], h_gpu)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, np.diff(off))
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, 180)
    for i in range(n):
        assert np.array_equal(np.sort(nnl[i, :noi[i]]), nbr[off[i]:off[i + 1]]), i
    left = np.abs(noi - 60) >= 5
    assert st["sml_out_of_band"] == int(left.sum())
    assert left.sum() < 0.005 * n and left.sum() < 0.02 * before
    assert (noi[left] <= 55).all() and np.array_equal(h_gpu[left], 2.0 * h_jacobi[left])
    sim.close()


@pytest.mark.parametrize("spread", [(0.7, 1.4), (2.0, 2.4)])
def test_variable_h_on_lists_matches_oracle(spread, cuda):
    """The variable-h iteration on neighbour lists: the final h equal to the
    oracle's Jacobi iteration from the same start, and every list and count
    equal to the brute-force set of the final h.  With h started 2-2.4x too
    large the first counts pass max_num_interactions (180): the lists are
    truncated and re-walked after each sweep, with the same result."""
    S, C = _cloud_state(20_000, spread=spread)
    n = len(S["x"])
    mat = material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)
    sim = Miluphpc(sph_cfg(variable_sml=1, integrate_energy=0), S, materials=[mat], want_nnl=True)
    sim.rhs(0)
    h_gpu = sim.numpy("sml")
    h_orc, _, _ = O.variable_h(S["x"], S["y"], S["z"], S["sml"], 60, tol=5, max_nb=180, max_iter=5)
    assert (np.abs(h_gpu - h_orc) <= 1e-12 * h_orc).mean() > 0.999
    off, nbr = O.frnn(S["x"], S["y"], S["z"], h_gpu)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, np.diff(off))
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, 180)
    for i in range(n):
        assert np.array_equal(np.sort(nnl[i, :noi[i]]), nbr[off[i]:off[i + 1]]), i
    st = sim.stats()
    assert st["max_noi"] == noi.max() and st["mean_noi"] == pytest.approx(noi.mean())
    sim.close()


@pytest.mark.parametrize("n", [1, 7, 100, 1000])
def test_variable_h_on_lists_small_n(n, cuda):
    """The list-based variable-h iteration and the band repair on a handful of
    particles (partial warps, a single tree leaf, counts far below the target):
    h equal to the oracle's iteration, lists equal to the brute-force sets."""
    S, C = _cloud_state(max(n, 2), seed=11)
    S = {k: (v[:n].copy() if isinstance(v, np.ndarray) and v.shape[:1] == (max(n, 2),) else v) for k, v in S.items()}
    mat = material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)
    sim = Miluphpc(sph_cfg(variable_sml=1, integrate_energy=0), S, materials=[mat], want_nnl=True)
    sim.rhs(0)
    h_gpu = sim.numpy("sml")
    h_orc, _, _ = O.variable_h(S["x"], S["y"], S["z"], S["sml"], 60, tol=5, max_nb=180, max_iter=5)
    assert (np.abs(h_gpu - h_orc) <= 1e-12 * h_orc).mean() > 0.99
    off, nbr = O.frnn(S["x"], S["y"], S["z"], h_gpu)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, np.diff(off))
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, 180)
    for i in range(n):
        assert np.array_equal(np.sort(nnl[i, :noi[i]]), nbr[off[i]:off[i + 1]]), i
    sim.close()


def test_variable_h_on_lists_after_steps(cuda):
    """The common case of the list-based iteration: a few steps into a run
    (band repair on), where most particles start in the band and the few
    that move edit the lists pair by pair.  One more right-hand side, band
    repair off, from the current state: h equal to the oracle's iteration from
    the same h, lists and counts equal to the brute-force sets."""
    S, C = _cloud_state(20_000)
    n = len(S["x"])
    mat = material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)
    cfg = sph_cfg(variable_sml=1, integrate_energy=0, sml_band_rounds=8, time_step=1e-3)
    sim = Miluphpc(cfg, S, materials=[mat], want_nnl=True)
    for k in range(3):
        sim.integrate(k)
    x, y, z, h0 = (sim.numpy(f) for f in ("x", "y", "z", "sml"))
    cfg.sml_band_rounds = 0
    sim.set_config(cfg)
    sim.rhs(3)
    h_gpu = sim.numpy("sml")
    h_orc, _, _ = O.variable_h(x, y, z, h0, 60, tol=5, max_nb=180, max_iter=5)
    assert (h_gpu != h0).sum() > 20  # some particles moved their h
    assert (np.abs(h_gpu - h_orc) <= 1e-12 * h_orc).mean() > 0.999
    off, nbr = O.frnn(x, y, z, h_gpu)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, np.diff(off))
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, 180)
    for i in range(n):
        assert np.array_equal(np.sort(nnl[i, :noi[i]]), nbr[off[i]:off[i + 1]]), i
    sim.close()


def test_run_totals_equal_per_step_counters(cuda):
    """The device-side run totals (run_* of mhpc_stats) equal the sums and the
    maximum of the per-RHS counters read after every step, and restart at
    mhpc_stats_reset_run."""
    S, C = _cloud_state(20_000)
    mat = material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)
    sim = Miluphpc(sph_cfg(variable_sml=1, integrate_energy=0, sml_band_rounds=2, time_step=1e-3), S,
                   materials=[mat])
    sim.integrate(0)
    sim.reset_run_stats()
    assert sim.stats()["run_rhs"] == 0
    per = []
    for k in range(1, 5):
        sim.integrate(k)
        per.append(sim.stats())
    tot = sim.stats()
    assert tot["run_rhs"] == 4 and tot["run_band_rhs"] == 4
    assert tot["run_out_of_band_sum"] == sum(s["sml_out_of_band"] for s in per)
    assert tot["run_out_of_band_max"] == max(s["sml_out_of_band"] for s in per)
    assert tot["run_band_before_sum"] == sum(s["sml_band_before"] for s in per)
    assert sum(s["sml_band_before"] for s in per) > 0
    assert tot["run_predictor_fallback_sum"] == sum(s["predictor_fallback"] for s in per)
    sim.reset_run_stats()
    sim.integrate(5)
    sim.integrate(6)
    assert sim.stats()["run_rhs"] == 2
    sim.close()


# ------------------------------------------------------ boundary checks
def test_boundary_argument_checks(cuda):
    P = ics.plummer(4096, seed=3)
    # h-tied softening needs every particle's h
    cfg = gravity_cfg(softening_mode=1, softening_h_factor=0.5)
    sim = Miluphpc(cfg, P)
    sim.soa.sml = None
    with pytest.raises(_lib.MhpcError) as e:
        sim.rhs(0)
    assert e.value.code == 1
    sim.close()
    # ... and with h it matches the direct sum with the same softening
    Q = dict(P)
    Q["sml"] = np.full(4096, 0.05)
    sim = Miluphpc(gravity_cfg(softening_mode=1, softening_h_factor=0.5, theta=1e-8), Q)
    sim.rhs(0)
    tg = np.arange(0, 4096, 64, dtype=np.int32)
    dx, dy, dz, _ = O.direct(P["x"], P["y"], P["z"], P["mass"], tg, 1e-4 + 0.025 ** 2)
    g = [sim.numpy(k)[tg] for k in ("g_ax", "g_ay", "g_az")]
    assert rel_err(*g, dx, dy, dz).max() < 1e-9
    # the creation config is accepted again (max_num_interactions 0 = 180)
    cfg0 = gravity_cfg(max_num_interactions=0)
    sim.set_config(cfg0)
    sim.close()
    # material ids outside the table are an argument error
    S = _sedov_state(12)
    S["material_id"] = np.zeros(len(S["x"]), dtype=np.int32)
    S["material_id"][5] = 3
    sim = Miluphpc(sph_cfg(), S, materials=[material()])
    with pytest.raises(_lib.MhpcError) as e:
        sim.rhs(0)
    assert e.value.code == 1
    sim.close()
