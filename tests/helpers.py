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
