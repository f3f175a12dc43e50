"""Seeded synthetic initial conditions for the benchmark workloads.

The reference reads its initial conditions from HDF5 files made by external
generators (Plummer: an external ParticleDistributor, Sedov:
testcases/sedov/initial_sedov.py).  Neither travels here, so these numpy
generators build inputs with the same shapes, sizes and distributions from a
recorded seed.  All arrays are float64 (the reference's `real`).
"""
import math

import numpy as np


def plummer(n, seed=1, a=1.0, rmax_over_a=10.0):
    """Plummer sphere, G = M = 1, scale radius a.

    Radii by inverse CDF r = a / sqrt(m^(-2/3) - 1) with m ~ U(0,1), redrawn
    while r >= rmax_over_a * a; isotropic directions; speeds q * v_esc(r),
    v_esc = sqrt(2) (1 + r^2/a^2)^(-1/4), with q drawn by von Neumann rejection
    on g(q) = q^2 (1 - q^2)^(7/2) (Aarseth, Henon & Wielen 1974).  Equal
    masses 1/n; centre of mass and mean velocity are removed.
    """
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        m = rng.uniform(0.0, 1.0, todo.size)
        m = np.clip(m, 1e-300, 1.0)
        rr = a / np.sqrt(m ** (-2.0 / 3.0) - 1.0)
        ok = rr < rmax_over_a * a
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    ct = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    st = np.sqrt(1.0 - ct * ct)
    x = r * st * np.cos(ph)
    y = r * st * np.sin(ph)
    z = r * ct
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        q0 = rng.uniform(0.0, 1.0, todo.size)
        g0 = rng.uniform(0.0, 0.1, todo.size)
        ok = g0 < q0 * q0 * (1.0 - q0 * q0) ** 3.5
        q[todo[ok]] = q0[ok]
        todo = todo[~ok]
    v = q * math.sqrt(2.0) * (1.0 + (r / a) ** 2) ** (-0.25)
    ct = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    st = np.sqrt(1.0 - ct * ct)
    vx = v * st * np.cos(ph)
    vy = v * st * np.sin(ph)
    vz = v * ct
    mass = np.full(n, 1.0 / n)
    for arr in (x, y, z, vx, vy, vz):
        arr -= arr.mean()
    return dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, mass=mass)


def cubic_w(r, h):
    """3-D cubic spline with support radius h (same kernel as the SPH path)."""
    q = r / h
    f = 8.0 / (math.pi * h ** 3)
    w = np.where(q > 1.0, 0.0,
                 np.where(q > 0.5, 2.0 * f * (1.0 - q) ** 3, f * (6.0 * q ** 3 - 6.0 * q ** 2 + 1.0)))
    return w


def sedov(nside=128, seed=2, jitter=1e-3, gamma=5.0 / 3.0, u0=1e-6, e_blast=1.0, h_factor=2.5):
    """Sedov blast on a cubic lattice of nside^3 cell centres in [-0.5, 0.5]^3.

    Positions jittered by U(-jitter, jitter) * dx, rho = 1 (m = 1/N), specific
    energy u0 everywhere plus e_blast spread over particles within r < 2h of
    the origin in proportion to the cubic-spline weight W(r, 2h); fixed
    smoothing length (support radius) h = h_factor * dx.
    """
    rng = np.random.default_rng(seed)
    dx = 1.0 / nside
    c = -0.5 + (np.arange(nside) + 0.5) * dx
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    x = xx.ravel().copy(); y = yy.ravel().copy(); z = zz.ravel().copy()
    n = x.size
    x += rng.uniform(-jitter, jitter, n) * dx
    y += rng.uniform(-jitter, jitter, n) * dx
    z += rng.uniform(-jitter, jitter, n) * dx
    h = h_factor * dx
    mass = np.full(n, 1.0 / n)
    r = np.sqrt(x * x + y * y + z * z)
    w = cubic_w(r, 2.0 * h)
    e = np.full(n, u0)
    sw = w.sum()
    e += e_blast * w / (sw * mass)
    zeros = np.zeros(n)
    return dict(x=x, y=y, z=z, vx=zeros.copy(), vy=zeros.copy(), vz=zeros.copy(), mass=mass,
                sml=np.full(n, h), e=e, rho=np.ones(n), gamma=gamma)


def rotating_cloud(n, seed=3, radius=1.0, e_rot_ratio=0.16, e_th_ratio=0.26, n_target=60,
                   perturbation=0.1):
    """Self-gravitating isothermal rotating cloud (G = M = R = 1).

    Uniform sphere with density rho0 (1 + perturbation cos 2 phi) by rejection
    sampling; solid-body rotation about z with E_rot / |E_grav| = e_rot_ratio
    (Omega^2 = 2 e_rot_ratio (3/5) / (2/5) for a uniform sphere); isothermal
    sound speed from E_th / |E_grav| = e_th_ratio with E_th = (3/2) M c_s^2.
    Initial smoothing length from the mean density for n_target neighbours.
    """
    rng = np.random.default_rng(seed)
    pos = np.empty((n, 3))
    got = 0
    while got < n:
        k = int((n - got) * 2.2) + 1024
        p = rng.uniform(-radius, radius, (k, 3))
        r2 = (p * p).sum(1)
        p = p[r2 < radius * radius]
        phi = np.arctan2(p[:, 1], p[:, 0])
        acc = rng.uniform(0.0, 1.0 + perturbation, p.shape[0]) < 1.0 + perturbation * np.cos(2 * phi)
        p = p[acc]
        take = min(n - got, p.shape[0])
        pos[got:got + take] = p[:take]
        got += take
    x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    e_grav = 3.0 / 5.0
    omega = math.sqrt(2.0 * e_rot_ratio * e_grav / (2.0 / 5.0))
    vx = -omega * y
    vy = omega * x
    vz = np.zeros(n)
    cs2 = e_th_ratio * e_grav / 1.5
    mass = np.full(n, 1.0 / n)
    h0 = radius * (n_target / n) ** (1.0 / 3.0)
    return dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, mass=mass, sml=np.full(n, h0),
                cs2=cs2, omega=omega, e=np.full(n, cs2), rho=np.full(n, 1.0 / (4.0 / 3.0 * math.pi)))
