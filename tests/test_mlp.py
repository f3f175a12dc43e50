"""The learned smoothing-length predictor.

CPU: the FP64 oracle's analytic backward pass agrees with central differences.
GPU: the tensor-core forward/backward kernels agree with the oracle (which
rounds to BF16 where the kernels do); training lowers the loss; and on a
rotating cloud the trained predictor lets most particles stop after the first
variable-h sweep, where the plain iteration needs more sweeps for them.
"""
import ctypes

import numpy as np
import pytest

from miluphpc_b200 import _lib, ics
from oracle import mlp_oracle as MO


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(MO.N_PARAM)
    W1 = rng.normal(0, 0.5, (MO.N_H, MO.N_INP))
    W1[:, MO.N_IN:] = 0
    p[MO.OFF_W1:MO.OFF_B1] = W1.ravel()
    p[MO.OFF_B1:MO.OFF_W2] = rng.normal(0, 0.1, MO.N_H)
    p[MO.OFF_W2:MO.OFF_B2] = rng.normal(0, 0.2, MO.N_H * MO.N_H)
    p[MO.OFF_B2:MO.OFF_W3] = rng.normal(0, 0.1, MO.N_H)
    p[MO.OFF_W3:MO.OFF_B3] = rng.normal(0, 0.3, MO.N_H)
    p[MO.OFF_B3] = 0.05
    return p


def test_oracle_backward_is_the_gradient():
    rng = np.random.default_rng(1)
    p = _rand_params(2)
    X = rng.normal(0, 1, (64, MO.N_IN))
    y = rng.normal(0, 1, 64)
    # unrounded analytic gradient vs central differences
    W1, b1, W2, b2, w3, b3 = MO.unpack(p)
    idx = [MO.OFF_W1 + 3, MO.OFF_B1 + 5, MO.OFF_W2 + 777, MO.OFF_B2 + 9, MO.OFF_W3 + 11, MO.OFF_B3]
    num = MO.numeric_grad(p, X, y, idx)
    # analytic without BF16 rounding: call with rounding disabled via exact inputs
    old = MO.bf16
    try:
        MO.bf16 = lambda a: np.asarray(a, dtype=np.float64)
        _, _, g = MO.forward_backward(p, X, y)
    finally:
        MO.bf16 = old
    np.testing.assert_allclose(g[idx], num, rtol=1e-5, atol=1e-9)


@pytest.mark.gpu
def test_mlp_forward_backward_matches_oracle(cuda):
    import torch
    from miluphpc_b200.miluphpc import Miluphpc, material
    C = ics.rotating_cloud(4096, seed=1)
    C["p"] = np.zeros(4096); C["cs"] = np.zeros(4096)
    cfg = _lib.default_config(gravity=0, sph=1, variable_sml=1, learned_h=1, integrator=0, time_step=1e-3)
    sim = Miluphpc(cfg, C, materials=[material(interactions=60, eos_type=0, K=0.104, gamma=1.0)])
    L = _lib.load()
    assert L.mhpc_mlp_num_params() == MO.N_PARAM
    p = _rand_params(3).astype(np.float32)
    _lib.check(L.mhpc_mlp_set_params(sim.ctx, p.ctypes.data_as(_lib.P_f)), "set_params")
    rng = np.random.default_rng(4)
    rows = 300
    X = rng.normal(0, 1, (rows, MO.N_IN)).astype(np.float32)
    y = rng.normal(0, 1, rows).astype(np.float32)
    tX = torch.as_tensor(X, device=cuda)
    ty = torch.as_tensor(y, device=cuda)
    out = torch.zeros(rows, dtype=torch.float32, device=cuda)
    grad = torch.zeros(MO.N_PARAM, dtype=torch.float32, device=cuda)
    loss = ctypes.c_float()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.check(L.mhpc_mlp_forward_backward(sim.ctx, vp(tX), rows, vp(ty), vp(out), vp(grad), ctypes.byref(loss)),
               "forward_backward")
    o_ref, l_ref, g_ref = MO.forward_backward(p.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    np.testing.assert_allclose(out.cpu().numpy(), o_ref, rtol=2e-3, atol=2e-3)
    assert abs(loss.value - l_ref) <= 2e-3 * l_ref
    g = grad.cpu().numpy()
    for lo, hi in ((MO.OFF_W1, MO.OFF_B1), (MO.OFF_B1, MO.OFF_W2), (MO.OFF_W2, MO.OFF_B2), (MO.OFF_B2, MO.OFF_W3),
                   (MO.OFF_W3, MO.OFF_B3 + 1)):
        ref = g_ref[lo:hi]
        err = np.linalg.norm(g[lo:hi] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 5e-3, (lo, err)
    sim.close()


def _cloud_sim(n, learned, seed=3, **kw):
    from miluphpc_b200.miluphpc import Miluphpc, material
    C = ics.rotating_cloud(n, seed=seed)
    C["p"] = np.zeros(n); C["cs"] = np.zeros(n)
    cfg = _lib.default_config(gravity=1, sph=1, variable_sml=1, learned_h=int(learned), integrator=0,
                              time_step=0.004, smoothing=0.0, softening_mode=1, softening_h_factor=0.5,
                              precision=1, theta_mixed=0.25, sfc=1, **kw)
    return Miluphpc(cfg, C, materials=[material(interactions=60, eos_type=0, K=C["cs2"], gamma=1.0)])


@pytest.mark.gpu
def test_training_lowers_loss_and_predictor_saves_sweeps(cuda):
    n = 65536
    sim = _cloud_sim(n, learned=True)
    plain = _cloud_sim(n, learned=False)
    L = _lib.load()
    for step in range(12):
        sim.integrate(step)
        plain.integrate(step)
    loss0 = ctypes.c_float()
    _lib.check(L.mhpc_mlp_train(sim.ctx, 1, 1e-3, ctypes.byref(loss0)), "train")
    loss1 = ctypes.c_float()
    _lib.check(L.mhpc_mlp_train(sim.ctx, 600, 1e-3, ctypes.byref(loss1)), "train")
    assert loss1.value < 0.5 * loss0.value, (loss0.value, loss1.value)
    fall_l, fall_p, band_l, band_p = [], [], [], []
    for step in range(12, 18):
        sim.integrate(step)
        plain.integrate(step)
        sl, sp = sim.stats(), plain.stats()
        fall_l.append(sl["predictor_fallback"])
        fall_p.append(sp["predictor_fallback"])
        band_l.append(sl["sml_out_of_band"])
        band_p.append(sp["sml_out_of_band"])
    # the first prediction is made from features of a plain step; from then on
    # fewer particles need a second sweep than with the plain iteration
    assert np.mean(fall_l[1:]) < 0.6 * np.mean(fall_p[1:]), (fall_l, fall_p)
    # and the final neighbour counts are no worse
    assert np.mean(band_l[1:]) <= 1.2 * np.mean(band_p[1:]) + 0.001 * n, (band_l, band_p)
    sim.close()
    plain.close()


def _params(sim):
    L = _lib.load()
    k = L.mhpc_mlp_num_params()
    buf = (ctypes.c_float * k)()
    _lib.check(L.mhpc_mlp_get_params(sim.ctx, buf), "get_params")
    return np.frombuffer(buf, dtype=np.float32).copy()


@pytest.mark.gpu
def test_predictor_refresh_between_steps(cuda):
    """Once trained, the predictor takes learned_refresh_iters Adam steps every
    learned_refresh_every right-hand sides (queued on the stream, no host
    synchronisation): its weights change at exactly those right-hand sides,
    and stay fixed when the refresh is off."""
    n = 32768
    L = _lib.load()
    runs = {}
    for every in (0, 3):
        sim = _cloud_sim(n, learned=True, learned_refresh_every=every, learned_refresh_iters=4)
        for step in range(12):
            sim.integrate(step)
        _lib.check(L.mhpc_mlp_train(sim.ctx, 50, 1e-3, None), "train")
        w = [_params(sim)]
        for step in range(12, 18):  # right-hand sides 13..18: refreshes at 15 and 18 when every = 3
            sim.integrate(step)
            w.append(_params(sim))
        runs[every] = w
        sim.close()
    fixed = runs[0]
    assert all(np.array_equal(fixed[0], x) for x in fixed[1:])
    moved = runs[3]
    changed = [not np.array_equal(moved[k], moved[k + 1]) for k in range(6)]
    assert changed == [False, False, True, False, False, True], changed
