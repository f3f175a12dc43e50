"""Oracle and CUDA path against milupHPC's own outputs.

The fixtures tests/golden/ref_*.npz hold seeded inputs and what the
reference's kernels returned for them (tests/golden/make_golden.py runs the
reference harness built from the reference sources):

* gravity (testcases/plummer/parameter.h build): computeBoundingBox, buildTree,
  calculateCentersOfMass, sortArray of the supplied SFC keys,
  computeForces_v2 -- src/subdomain_key_tree/tree.cu:302-437, 768-1083,
  1416-1480; src/helper.cu:150-166; src/gravity/gravity.cu:726-903.
* SPH (testcases/sedov/parameter.h build: ideal gas, INTEGRATE_ENERGY,
  INTEGRATE_SML, cubic spline): fixedRadiusNN v0, calculateDensity,
  calculateSoundSpeed, calculatePressure, internalForces --
  src/sph/sph.cu:93-281, src/sph/density.cu, src/sph/soundspeed.cu,
  src/sph/pressure.cu, src/sph/internal_forces.cu.

Bars: bounding box, tree cells (key prefix, level), every particle's path and
the sorted order exact; centres of mass exact; forces within 1e-12 relative
(the reference takes CUDA's rsqrt, the oracle 1/sqrt); neighbour sets equal;
density, pressure, sound speed within 1e-12; SPH rates within 1e-10 of their
largest magnitude (the neighbour order, hence the summation order, differs).
"""
import importlib.util
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GRAVITY = ["ref_gravity_lebesgue", "ref_gravity_hilbert"]


def fixture(name):
    path = os.path.join(GOLDEN, name + ".npz")
    assert os.path.exists(path), "missing reference fixture " + path
    return dict(np.load(path))


def tree_walk(child, n, x, y, z, m):
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.walk_ref_tree(child, n, x, y, z, m)


def close_rates(got, ref, tol=1e-10):
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= tol * scale, (np.abs(got - ref).max(), scale)


# ----------------------------------------------------------------- oracle --
@pytest.mark.parametrize("name", GRAVITY)
def test_oracle_tree_and_v2_match_reference(name):
    F = fixture(name)
    x, y, z, m = F["x"], F["y"], F["z"], F["m"]
    n = len(x)
    bb = O.bbox(x, y, z)
    assert np.array_equal(bb, F["bbox"])
    # each particle's path through the reference tree is its Lebesgue key prefix
    lk = O.keys(x, y, z, bb, 0)
    shift = (3 * (21 - F["leaf_level"].astype(np.int64))).astype(np.uint64)
    assert np.array_equal(lk >> shift, F["leaf_prefix"])
    T = O.Tree(x, y, z, m, bb)
    assert T.nodes - n == int(F["cells"])
    cp, cl, com, lp, ll = tree_walk(T.child, n, T.x, T.y, T.z, T.m)
    assert np.array_equal(cp, F["cell_prefix"]) and np.array_equal(cl, F["cell_level"])
    assert np.array_equal(lp, F["leaf_prefix"]) and np.array_equal(ll, F["leaf_level"])
    assert np.array_equal(com, F["cell_com"])
    keys = O.keys(x, y, z, bb, int(F["curve"]))
    _, perm = O.sort(keys)
    assert np.array_equal(perm, F["sorted"])
    ax, ay, az = O.gravity_v2(T, perm, 0.5 * (bb[1] - bb[0]), float(F["theta"]), float(F["eps2"]))
    e = rel_err(ax, ay, az, F["ax"], F["ay"], F["az"])
    assert e.max() < 1e-12, e.max()


def test_oracle_sph_matches_reference():
    F = fixture("ref_sph")
    x, y, z, m, h = F["x"], F["y"], F["z"], F["m"], F["sml"]
    assert np.array_equal(O.bbox(x, y, z), F["bbox"])
    off, nbr = O.frnn(x, y, z, h)
    noi = np.diff(off)
    assert np.array_equal(noi, F["noi"])
    owner = np.repeat(np.arange(len(x)), noi)
    nb = nbr.astype(np.int64)
    assert np.array_equal(np.bincount(owner, weights=nb, minlength=len(x)).astype(np.int64), F["nb_sum"])
    assert np.array_equal(np.bincount(owner, weights=nb * nb, minlength=len(x)).astype(np.int64), F["nb_sq"])
    # INTEGRATE_SML: kernels of a pair use the mean smoothing length
    rho = O.density(x, y, z, m, h, off, nbr, avg_h=True)
    np.testing.assert_allclose(rho, F["rho"], rtol=1e-12)
    p, cs = O.eos(9, np.array([0.0, float(F["gamma"]), 0.0, 0.0, 0.0]), rho, F["e"], F["p"])
    np.testing.assert_allclose(p, F["p_out"], rtol=1e-12)
    np.testing.assert_allclose(cs, F["cs_out"], rtol=1e-12)
    ax, ay, az, drho, de, dh = O.forces(x, y, z, F["vx"], F["vy"], F["vz"], m, h, rho, p, cs, off, nbr,
                                        float(F["alpha"]), float(F["beta"]), avg_h=True,
                                        integrate_sml=True)
    for got, ref in ((ax, F["ax"]), (ay, F["ay"]), (az, F["az"]), (drho, F["drhodt"]), (de, F["dedt"]),
                     (dh, F["dsmldt"])):
        close_rates(got, ref)


def test_oracle_balsara_matches_reference():
    """Balsara switch (harness build with BALSARA_SWITCH on): div v, curl v of
    CalcDivvandCurlv and the switched viscosity of internalForces."""
    F = fixture("ref_sph_balsara")
    x, y, z, m, h = F["x"], F["y"], F["z"], F["m"], F["sml"]
    off, nbr = O.frnn(x, y, z, h)
    assert np.array_equal(np.diff(off), F["noi"])
    rho = O.density(x, y, z, m, h, off, nbr, avg_h=True)
    np.testing.assert_allclose(rho, F["rho"], rtol=1e-12)
    p, cs = O.eos(9, np.array([0.0, float(F["gamma"]), 0.0, 0.0, 0.0]), rho, F["e"], F["p"])
    # INTEGRATE_SML without VARIABLE_SML: the gradients use h_i
    divv, curl, f = O.balsara(x, y, z, F["vx"], F["vy"], F["vz"], m, h, rho, cs, off, nbr, avg_h=False)
    close_rates(divv, F["divv"])
    close_rates(curl, F["curlv"])
    ax, ay, az, drho, de, dh = O.forces(x, y, z, F["vx"], F["vy"], F["vz"], m, h, rho, p, cs, off, nbr,
                                        float(F["alpha"]), float(F["beta"]), avg_h=True, integrate_sml=True,
                                        bal=f)
    for got, ref in ((ax, F["ax"]), (ay, F["ay"]), (az, F["az"]), (drho, F["drhodt"]), (de, F["dedt"]),
                     (dh, F["dsmldt"])):
        close_rates(got, ref)
    # the switch changes the answer: without it the viscous terms differ
    ax0 = O.forces(x, y, z, F["vx"], F["vy"], F["vz"], m, h, rho, p, cs, off, nbr, float(F["alpha"]),
                   float(F["beta"]), avg_h=True, integrate_sml=True)[0]
    assert np.abs(ax0 - F["ax"]).max() > 1e-6 * np.abs(F["ax"]).max()


# -------------------------------------------------------------- CUDA path --
@pytest.mark.gpu
@pytest.mark.parametrize("name", GRAVITY)
def test_cuda_gravity_matches_reference(name, cuda):
    from miluphpc_b200.miluphpc import Miluphpc
    from tests.helpers import gravity_cfg
    F = fixture(name)
    n = len(F["x"])
    P = dict(x=F["x"], y=F["y"], z=F["z"], mass=F["m"], vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n))
    cfg = gravity_cfg(sfc=int(F["curve"]), theta=float(F["theta"]), smoothing=float(F["eps2"]))
    sim = Miluphpc(cfg, P)
    sim.rhs(0)
    _, perm = sim.export_sorted()
    assert np.array_equal(perm, F["sorted"])
    tr = sim.export_tree(2 * n + 20000)
    assert tr["cells"] == int(F["cells"])
    cp, cl, com, lp, ll = tree_walk(tr["child"], n, tr["x"], tr["y"], tr["z"], tr["m"])
    assert np.array_equal(cp, F["cell_prefix"]) and np.array_equal(cl, F["cell_level"])
    assert np.array_equal(lp, F["leaf_prefix"]) and np.array_equal(ll, F["leaf_level"])
    if int(F["curve"]) == 0:
        assert np.array_equal(com, F["cell_com"])
    else:
        np.testing.assert_allclose(com, F["cell_com"], rtol=1e-12, atol=1e-14)
    e = rel_err(sim.numpy("g_ax"), sim.numpy("g_ay"), sim.numpy("g_az"), F["ax"], F["ay"], F["az"])
    assert e.max() < 1e-9, e.max()
    sim.close()


@pytest.mark.gpu
def test_cuda_sph_matches_reference(cuda):
    from miluphpc_b200.miluphpc import Miluphpc, material
    from tests.helpers import sph_cfg
    F = fixture("ref_sph")
    n = len(F["x"])
    S = {k: F[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "sml", "e", "p", "cs")}
    S["mass"] = F["m"].copy()
    cfg = sph_cfg(integrate_sml=1)
    mat = material(interactions=50, alpha=float(F["alpha"]), beta=float(F["beta"]), eos_type=9,
                   gamma=float(F["gamma"]))
    sim = Miluphpc(cfg, S, materials=[mat], want_nnl=True)
    sim.rhs(0)
    noi = sim.numpy("noi")
    assert np.array_equal(noi, F["noi"])
    nnl = sim.t["nnl"].cpu().numpy().reshape(n, cfg.max_num_interactions).astype(np.int64)
    mask = np.arange(cfg.max_num_interactions)[None, :] < noi[:, None]
    assert np.array_equal(np.where(mask, nnl, 0).sum(1), F["nb_sum"])
    assert np.array_equal(np.where(mask, nnl * nnl, 0).sum(1), F["nb_sq"])
    np.testing.assert_allclose(sim.numpy("rho"), F["rho"], rtol=1e-12)
    np.testing.assert_allclose(sim.numpy("p"), F["p_out"], rtol=1e-12)
    np.testing.assert_allclose(sim.numpy("cs"), F["cs_out"], rtol=1e-12)
    for k, ref in (("ax", "ax"), ("ay", "ay"), ("az", "az"), ("drhodt", "drhodt"), ("dedt", "dedt"),
                   ("dsmldt", "dsmldt")):
        close_rates(sim.numpy(k), F[ref])
    sim.close()


@pytest.mark.gpu
def test_cuda_balsara_matches_reference(cuda):
    from miluphpc_b200.miluphpc import Miluphpc, material
    from tests.helpers import sph_cfg
    F = fixture("ref_sph_balsara")
    S = {k: F[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "sml", "e", "p", "cs")}
    S["mass"] = F["m"].copy()
    cfg = sph_cfg(integrate_sml=1, balsara=1)
    mat = material(interactions=50, alpha=float(F["alpha"]), beta=float(F["beta"]), eos_type=9,
                   gamma=float(F["gamma"]))
    sim = Miluphpc(cfg, S, materials=[mat])
    sim.rhs(0)
    assert np.array_equal(sim.numpy("noi"), F["noi"])
    np.testing.assert_allclose(sim.numpy("rho"), F["rho"], rtol=1e-12)
    for k in ("ax", "ay", "az", "drhodt", "dedt", "dsmldt"):
        close_rates(sim.numpy(k), F[k])
    sim.close()


# ------------------------------------------------------------ Hilbert keys --
# ref_hilbert.npz: Lebesgue keys (seeded random 63-bit keys, a seeded Plummer
# sphere's keys, edge keys) and their Hilbert keys from the reference's own
# KeyNS::lebesgue2hilbert(key, 21, 21) (src/subdomain_key_tree/tree.cu:40-53,
# the conversion of Tree::getParticleKey, tree.cu:233), run on the CPU.
def test_oracle_hilbert_matches_reference():
    F = fixture("ref_hilbert")
    got = np.array([O.lebesgue2hilbert(int(k)) for k in F["lebesgue"]], dtype=np.uint64)
    assert np.array_equal(got, F["hilbert"])


@pytest.mark.gpu
def test_gpu_hilbert_keys_match_reference(cuda):
    """The CUDA key kernel (curve 1) on the Plummer positions of the fixture
    equals the reference's conversion of the same positions' Lebesgue keys."""
    from tests.test_gpu_parity import gpu_keys
    F = fixture("ref_hilbert")
    a, b = int(F["n_random"]), int(F["n_random"] + F["n_plummer"])
    _, leb = gpu_keys(F["x"], F["y"], F["z"], 0)
    assert np.array_equal(leb, F["lebesgue"][a:b])
    _, hil = gpu_keys(F["x"], F["y"], F["z"], 1)
    assert np.array_equal(hil, F["hilbert"][a:b])


# ------------------------------------------------------------- integrators --
# ref_integrators.npz: a seeded random state and what milupHPC's own update
# kernels made of it (Sedov parameter.h build: INTEGRATE_ENERGY, INTEGRATE_SML,
# no INTEGRATE_DENSITY): ExplicitEulerNS::Kernel::update, LeapfrogNS::Kernel::
# updateX / updateV and PredictorCorrectorEulerNS::Kernel::predictor /
# corrector (src/integrator/device_explicit_euler.cu:4-54,
# device_leapfrog.cu:4-58, device_predictor_corrector_euler.cu:130-300).
# The reference build rounds every product and sum (-fmad=false), so the bar
# is bit-identical.
def _integ():
    F = fixture("ref_integrators")
    st = {k[3:]: F[k] for k in F if k.startswith("in_")}
    return F, st, float(F["dt"])


def _pc_numpy(st, dt):
    """The predictor and corrector formulas in elementwise IEEE double."""
    q = {}
    for c, v, a, g in (("x", "vx", "ax", "g_ax"), ("y", "vy", "ay", "g_ay"), ("z", "vz", "az", "g_az")):
        q[c] = st[c] + dt * st[v]
        q[v] = st[v] + dt * (st[a] + st[g])
    q["e"] = np.maximum(st["e"] + dt * st["dedt"], 1e-6)
    q["sml"], q["cs"], q["p"] = st["sml"], st["cs"], st["p"]
    return q


def test_oracle_integrators_match_reference():
    F, st, dt = _integ()
    e = O.euler(st, dt, gravity=True, sph=True, integrate_energy=True, integrate_sml=True)
    for k in ("x", "y", "z", "vx", "vy", "vz", "e", "sml"):
        assert np.array_equal(e[k], F["euler_" + k]), k
    ref = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("g_ax_old", "g_ay_old", "g_az_old"):
        ref[k] = np.zeros_like(ref["x"])
    p = O._p
    O.lib().orc_leapfrog_x(len(ref["x"]), dt, *[p(ref[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "g_ax", "g_ay",
                                                                     "g_az", "g_ax_old", "g_ay_old", "g_az_old")])
    for k in ("x", "y", "z", "g_ax_old", "g_ay_old", "g_az_old"):
        assert np.array_equal(ref[k], F["leapfrog_" + k]), k
    ref["g_ax"], ref["g_ay"], ref["g_az"] = st["gx2"], st["gy2"], st["gz2"]
    O.lib().orc_leapfrog_v(len(ref["x"]), dt, *[p(np.ascontiguousarray(ref[k])) for k in (
        "vx", "vy", "vz", "g_ax", "g_ay", "g_az", "g_ax_old", "g_ay_old", "g_az_old")])
    # orc_leapfrog_v updated ref's own velocity arrays in place
    for k in ("vx", "vy", "vz"):
        assert np.array_equal(ref[k], F["leapfrog_" + k]), k
    q = _pc_numpy(st, dt)
    for k in ("x", "y", "z", "vx", "vy", "vz", "e", "sml", "cs", "p"):
        assert np.array_equal(q[k], F["predictor_" + k]), k
    h = 0.5 * dt
    pde, pdh = 0.5 * st["dedt"], 0.5 * st["dsmldt"]
    for c, v, a, g, pa in (("x", "vx", "ax", "g_ax", "pax"), ("y", "vy", "ay", "g_ay", "pay"),
                           ("z", "vz", "az", "g_az", "paz")):
        assert np.array_equal(st[c] + h * (q[v] + st[v]), F["corrector_" + c]), c
        assert np.array_equal(st[v] + h * ((st[pa] + st[a]) + 2 * st[g]), F["corrector_" + v]), v
        assert np.array_equal(0.5 * (st[pa] + st[a]) + st[g], F["corrector_" + a]), a
    assert np.array_equal(np.maximum(st["e"] + h * (pde + st["dedt"]), 1e-6), F["corrector_e"])
    assert np.array_equal(0.5 * (pde + st["dedt"]), F["corrector_dedt"])
    assert np.array_equal(st["sml"] + h * (pdh + st["dsmldt"]), F["corrector_sml"])
    assert np.array_equal(0.5 * (pdh + st["dsmldt"]), F["corrector_dsmldt"])


@pytest.mark.gpu
def test_gpu_integrators_match_reference(cuda):
    """The library's update kernels through mhpc_integrate_euler /
    _leapfrog / _pc_predictor / _pc_corrector, bit for bit."""
    import ctypes
    import torch
    from miluphpc_b200 import _lib
    from miluphpc_b200.miluphpc import Miluphpc, material
    from tests.helpers import sph_cfg
    F, st, dt = _integ()
    L = _lib.load()
    n = len(st["x"])
    cfg = sph_cfg(gravity=1, integrator=1, integrate_energy=1, integrate_sml=1, integrate_density=0,
                  max_time_step=1.0)
    mat = [material(eos_type=9)]
    sim = Miluphpc(cfg, st, materials=mat)
    _lib.check(L.mhpc_integrate_euler(sim.ctx, ctypes.byref(sim.soa), dt), "euler")
    torch.cuda.synchronize()
    for k in ("x", "y", "z", "vx", "vy", "vz", "e", "sml"):
        assert np.array_equal(sim.numpy(k), F["euler_" + k]), k
    sim.close()
    sim = Miluphpc(cfg, st, materials=mat)
    _lib.check(L.mhpc_integrate_leapfrog(sim.ctx, ctypes.byref(sim.soa), dt, 0), "leapfrog x")
    for k, g in (("g_ax", "gx2"), ("g_ay", "gy2"), ("g_az", "gz2")):
        sim.t[k][:n] = torch.as_tensor(st[g], device=cuda)
    _lib.check(L.mhpc_integrate_leapfrog(sim.ctx, ctypes.byref(sim.soa), dt, 1), "leapfrog v")
    torch.cuda.synchronize()
    for k in ("x", "y", "z", "g_ax_old", "g_ay_old", "g_az_old", "vx", "vy", "vz"):
        assert np.array_equal(sim.numpy(k), F["leapfrog_" + k]), k
    sim.close()
    sim = Miluphpc(cfg, st, materials=mat)
    q = Miluphpc(cfg, {k: np.zeros(n) for k in ("x",)}, materials=mat)
    dt_dev = torch.full((1,), dt, dtype=torch.float64, device=cuda)
    _lib.check(L.mhpc_integrate_pc_predictor(sim.ctx, ctypes.byref(sim.soa), ctypes.byref(q.soa),
                                             ctypes.c_void_p(dt_dev.data_ptr())), "predictor")
    torch.cuda.synchronize()
    for k in ("x", "y", "z", "vx", "vy", "vz", "e", "sml", "cs", "p"):
        assert np.array_equal(q.numpy(k), F["predictor_" + k]), k
    for k, v in (("ax", st["pax"]), ("ay", st["pay"]), ("az", st["paz"]), ("dedt", 0.5 * st["dedt"]),
                 ("dsmldt", 0.5 * st["dsmldt"]), ("drhodt", st["drhodt"])):
        q.t[k][:n] = torch.as_tensor(v, device=cuda)
    _lib.check(L.mhpc_integrate_pc_corrector(sim.ctx, ctypes.byref(sim.soa), ctypes.byref(q.soa),
                                             ctypes.c_void_p(dt_dev.data_ptr())), "corrector")
    torch.cuda.synchronize()
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "e", "dedt", "sml", "dsmldt"):
        assert np.array_equal(sim.numpy(k), F["corrector_" + k]), k
    sim.close()
    q.close()
