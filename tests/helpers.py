"""Shared helpers of the parity tests: build workloads, run the GPU path
through the C ABI, run the oracle on the same inputs."""
import ctypes

import numpy as np

from miluphpc_b200 import _lib, ics


def plummer_state(n, seed=1):
    return ics.plummer(n, seed=seed)


def gravity_cfg(**kw):
    base = dict(gravity=1, sph=0, integrator=2, time_step=0.025, theta=0.5, smoothing=1e-4, sfc=0)
    base.update(kw)
    return _lib.default_config(**base)


def sph_cfg(**kw):
    base = dict(gravity=0, sph=1, integrator=0, time_step=1e-4, smoothing_kernel=1, integrate_energy=1,
                integrate_density=0, integrate_sml=0, variable_sml=0, max_num_interactions=180)
    base.update(kw)
    return _lib.default_config(**base)


def rel_err(ax, ay, az, bx, by, bz):
    num = np.sqrt((ax - bx) ** 2 + (ay - by) ** 2 + (az - bz) ** 2)
    den = np.sqrt(bx ** 2 + by ** 2 + bz ** 2)
    return num / np.maximum(den, 1e-300)


def nodeset_pairs(prefixes, levels):
    return set(zip((int(p) for p in prefixes), (int(l) for l in levels)))


def sedov_small(nside=24, seed=5):
    return ics.sedov(nside=nside, seed=seed)


def oracle_sph_rhs(O, S, alpha=1.0, beta=2.0, gamma=5.0 / 3.0, integrate_energy=True):
    """Miluphpc::parallel_sph on the oracle (fixed h, ideal gas): neighbours,
    density, sound speed from the previous pressure, pressure, forces."""
    off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr)
    p, cs = O.eos(9, np.array([0.0, gamma, 0.0, 0.0, 0.0]), rho, S["e"], S["p"])
    ax, ay, az, drho, de, dh = O.forces(S["x"], S["y"], S["z"], S["vx"], S["vy"], S["vz"], S["mass"], S["sml"],
                                        rho, p, cs, off, nbr, alpha, beta, integrate_energy=integrate_energy)
    return dict(rho=rho, p=p, cs=cs, ax=ax, ay=ay, az=az, drhodt=drho, dedt=de, noi=np.diff(off))


def oracle_pc_step(O, S, dt_max, time_left=1e30, alpha=1.0, beta=2.0, gamma=5.0 / 3.0):
    """One PredictorCorrectorEuler step (SPH only, fixed h, integrate energy)
    on the oracle: rhs, setTimeStep, predictor, rhs(predicted), corrector."""
    r = oracle_sph_rhs(O, S, alpha, beta, gamma)
    S = dict(S)
    S.update(rho=r["rho"], p=r["p"], cs=r["cs"])
    a2 = r["ax"] ** 2 + r["ay"] ** 2 + r["az"] ** 2
    with np.errstate(divide="ignore"):
        forces = np.min(np.sqrt(S["sml"] / np.sqrt(a2)))
        courant = np.min(S["sml"] / r["cs"])
        visc = np.min(0.4 * S["sml"] / (r["cs"] + 1.2 * alpha * r["cs"]))
    vmax = np.sqrt(S["vx"] ** 2 + S["vy"] ** 2 + S["vz"] ** 2).max()
    dt = min(0.4 * courant, 0.2 * forces)
    sr = 2 * S["sml"].max()
    if vmax > 0:
        dt = min(dt, sr / (2 * vmax))
    dt = min(dt, visc, time_left, dt_max)
    Q = dict(S)
    for c, a in (("x", "vx"), ("y", "vy"), ("z", "vz")):
        Q[c] = S[c] + dt * S[a]
    Q["vx"] = S["vx"] + dt * r["ax"]; Q["vy"] = S["vy"] + dt * r["ay"]; Q["vz"] = S["vz"] + dt * r["az"]
    Q["e"] = np.maximum(S["e"] + dt * r["dedt"], 1e-6)
    q = oracle_sph_rhs(O, Q, alpha, beta, gamma)
    N = dict(S)
    h = 0.5 * dt
    for c, v, a in (("x", "vx", "ax"), ("y", "vy", "ay"), ("z", "vz", "az")):
        N[c] = S[c] + h * (Q[v] + S[v])
        N[v] = S[v] + h * (q[a] + r[a])
    N["e"] = np.maximum(S["e"] + h * (q["dedt"] + r["dedt"]), 1e-6)
    # p and c_s keep the values of the first RHS (the second one wrote the
    # predicted state's copies)
    N["p"] = r["p"]
    N["cs"] = r["cs"]
    return N, dt
