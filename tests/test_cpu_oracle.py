"""CPU tests: pin the oracle with known answers and invariants, check the
host-side parsers and that libmhpc exports every symbol of include/mhpc.h.

The reference has no test suite and no golden vectors of its own.  The oracle
is pinned here by (a) closed-form known answers of the key construction
(bit layout, below-midpoint convention, Hilbert curve adjacency), (b) the
reference's own tree invariant `test_localTree` (tree.cu:1983-2080: node mass
= sum of children, COM consistent), (c) the limit theta -> 0 of the tree walk
equalling direct summation, and (d) the golden fixtures produced by running
the reference's own kernels (tests/test_ref_golden.py).
"""
import ctypes
import os
import re

import numpy as np
import pytest

from miluphpc_b200 import _lib, ics
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_key_bit_layout_known_answer():
    # box [-1, 1]^3; a point below the midpoint on all axes at every level is
    # the all-ones key; above everywhere is 0
    bb = np.array([-1.0, 1.0, -1.0, 1.0, -1.0, 1.0])
    lo = np.array([-0.9999999]); hi = np.array([0.9999999])
    k = O.keys(lo, lo, lo, bb, 0)
    assert int(k[0]) == (1 << 63) - 1
    k = O.keys(hi, hi, hi, bb, 0)
    assert int(k[0]) == 0
    # x below, y,z above at level 0 only -> octant 1 in the top digit
    k = O.keys(np.array([-0.5]), np.array([0.5]), np.array([0.5]), bb, 0)
    assert int(k[0]) >> 60 == 1
    # the midpoint itself is not below: son bit clear
    k = O.keys(np.array([0.0]), np.array([-0.1]), np.array([0.1]), bb, 0)
    assert (int(k[0]) >> 60) == 2


def test_hilbert_is_a_face_adjacent_curve():
    # level-3 cells ordered by Hilbert key must step to a face neighbour each
    # time: a property of the Hilbert curve that pins the reference's tables
    L = 3
    n = 2 ** L
    cells = []
    for ix in range(n):
        for iy in range(n):
            for iz in range(n):
                leb = 0
                for lvl in range(L):
                    sh = L - 1 - lvl
                    son = 0
                    # "below" = bit set: index from the top of the box
                    if not (ix >> sh) & 1:
                        son |= 1
                    if not (iy >> sh) & 1:
                        son |= 2
                    if not (iz >> sh) & 1:
                        son |= 4
                    leb = (leb << 3) | son
                full = leb << (3 * (21 - L))
                h = O.lebesgue2hilbert(full) >> (3 * (21 - L))
                cells.append((h, ix, iy, iz))
    cells.sort()
    assert [c[0] for c in cells] == list(range(n ** 3))
    for a, b in zip(cells, cells[1:]):
        assert abs(a[1] - b[1]) + abs(a[2] - b[2]) + abs(a[3] - b[3]) == 1


def test_bbox_contains_origin_and_is_cubic():
    x = np.array([1.0, 2.0]); y = np.array([3.0, 4.0]); z = np.array([0.5, 5.0])
    bb = O.bbox(x, y, z)
    assert list(bb) == [0.0, 5.0, 0.0, 5.0, 0.0, 5.0]


def test_sort_stable_on_ties():
    k = np.array([5, 3, 5, 1, 3, 5], dtype=np.uint64)
    ks, perm = O.sort(k)
    assert list(perm) == [3, 1, 4, 0, 2, 5]


@pytest.mark.parametrize("n", [2, 3, 500, 20000])
def test_tree_invariants_local_tree(n):
    P = ics.plummer(max(n, 2), seed=n)
    x, y, z, m = P["x"][:n], P["y"][:n], P["z"][:n], P["mass"][:n]
    bb = O.bbox(x, y, z)
    T = O.Tree(x, y, z, m, bb)
    # reference invariant test_localTree: mass of a node = sum of its children
    for node in range(n, T.nodes):
        ch = T.child[8 * node:8 * node + 8]
        ch = ch[ch >= 0]
        assert len(ch) >= 1
        assert abs(T.m[node] - T.m[ch].sum()) <= 1e-12 * T.m[node]
        com = (T.x[ch] * T.m[ch]).sum() / T.m[ch].sum()
        assert abs(T.x[node] - com) <= 1e-12 * max(1.0, abs(com))
    # every particle reachable exactly once
    seen = np.zeros(n, dtype=int)
    stack = [c for c in T.child[:8] if c >= 0]
    while stack:
        c = stack.pop()
        if c < n:
            seen[c] += 1
        else:
            stack.extend(cc for cc in T.child[8 * c:8 * c + 8] if cc >= 0)
    assert (seen == 1).all()


def test_node_set_is_the_prefix_set():
    # a cell (prefix, level) exists iff >= 2 particles share the prefix
    n = 3000
    P = ics.plummer(n, seed=4)
    bb = O.bbox(P["x"], P["y"], P["z"])
    T = O.Tree(P["x"], P["y"], P["z"], P["mass"], bb)
    pre, lev = T.nodeset()
    k = O.keys(P["x"], P["y"], P["z"], bb, 0)
    expect = set()
    for L in range(1, 22):
        p = k >> np.uint64(3 * (21 - L))
        u, c = np.unique(p, return_counts=True)
        expect |= {(int(a), L) for a in u[c >= 2]}
    assert set(zip(pre.tolist(), lev.tolist())) == expect


def test_walk_small_theta_is_direct_sum():
    n = 3000
    P = ics.plummer(n, seed=6)
    bb = O.bbox(P["x"], P["y"], P["z"])
    T = O.Tree(P["x"], P["y"], P["z"], P["mass"], bb)
    ax, ay, az, _ = O.gravity_v1(T, 0.5 * (bb[1] - bb[0]), 1e-6, 1e-4)
    dx, dy, dz, _ = O.direct(P["x"], P["y"], P["z"], P["mass"], np.arange(n), 1e-4)
    np.testing.assert_allclose(ax, dx, rtol=1e-9, atol=1e-12)
    _, perm = O.sort(O.keys(P["x"], P["y"], P["z"], bb, 0))
    bx, by, bz = O.gravity_v2(T, perm, 0.5 * (bb[1] - bb[0]), 1e-8, 1e-4)
    np.testing.assert_allclose(bx, dx, rtol=1e-9, atol=1e-12)


def test_relative_rule_floor_bounds_a_vanishing_acceleration():
    """Relative opening rule: a particle whose previous |a| is zero (the
    potential minimum) does not make its group open the whole tree; the
    sub-box's smallest |a| is floored at a tenth of its largest, so the
    group's interactions grow by a bounded factor and no other group changes."""
    n = 65_536
    P = ics.plummer(n, seed=2)
    bb = O.bbox(P["x"], P["y"], P["z"])
    radius = 0.5 * (bb[1] - bb[0])
    _, perm = O.sort(O.keys(P["x"], P["y"], P["z"], bb, 1))
    T = O.Tree(P["x"], P["y"], P["z"], P["mass"], bb)
    q = O.quad(T)
    ax, ay, az, _, _ = O.gravity_boxes(T, perm, radius, 0.28, 1e-4, q)
    amag = np.sqrt(ax ** 2 + ay ** 2 + az ** 2)
    _, _, _, c0, _ = O.gravity_boxes_rel(T, perm, radius, 1.0, 1e-4, q, amag, 1.8e-3)
    s = int(perm[1000])  # sorted position 1000: group 15, sub-box 5
    a2 = amag.copy()
    a2[s] = 0.0
    _, _, _, c1, _ = O.gravity_boxes_rel(T, perm, radius, 1.0, 1e-4, q, a2, 1.8e-3)
    grp = perm[960:1024]
    others = np.setdiff1d(np.arange(n), grp)
    assert np.array_equal(c1[others], c0[others])
    assert c1[s] >= c0[s] and c1[s] < 6 * c0[s], (c0[s], c1[s])
    assert c1[s] < n // 4


def test_frnn_equals_bruteforce():
    rng = np.random.default_rng(3)
    n = 1500
    x, y, z = rng.uniform(-1, 1, (3, n))
    h = rng.uniform(0.1, 0.3, n)
    off, nbr = O.frnn(x, y, z, h)
    d2 = (x[:, None] - x[None]) ** 2 + (y[:, None] - y[None]) ** 2 + (z[:, None] - z[None]) ** 2
    ok = (d2 < h[:, None] ** 2) & (d2 < h[None] ** 2)
    np.fill_diagonal(ok, False)
    for i in range(n):
        assert np.array_equal(nbr[off[i]:off[i + 1]], np.nonzero(ok[i])[0])


def test_density_of_uniform_lattice():
    S = ics.sedov(nside=16, seed=1, jitter=0.0)
    off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr)
    # interior particles of a unit-density lattice sum to ~1
    r = np.maximum.reduce([np.abs(S["x"]), np.abs(S["y"]), np.abs(S["z"])])
    inner = r < 0.5 - S["sml"][0]
    assert abs(rho[inner].mean() - 1.0) < 0.02


def test_forces_momentum_conservation():
    S = ics.sedov(nside=12, seed=2)
    n = len(S["x"])
    rng = np.random.default_rng(1)
    v = rng.normal(0, 0.1, (3, n))
    off, nbr = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    rho = O.density(S["x"], S["y"], S["z"], S["mass"], S["sml"], off, nbr)
    p, cs = O.eos(0, np.array([1.0, 1.4, 0, 0, 0]), rho, S["e"], np.zeros(n))
    ax, ay, az, drho, de, dh = O.forces(S["x"], S["y"], S["z"], v[0], v[1], v[2], S["mass"], S["sml"], rho, p,
                                        cs, off, nbr, 1.0, 2.0)
    # symmetric pair forces with equal h: total momentum change is zero
    tot = np.abs((S["mass"] * ax).sum()) + np.abs((S["mass"] * ay).sum())
    assert tot < 1e-10 * np.abs(S["mass"] * ax).sum()


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "mhpc.h")).read()
    declared = set(re.findall(r"\b(mhpc_[a-z_0-9]+)\s*\(", header))
    L = _lib.load()
    for name in declared:
        assert hasattr(L, name), name
    assert declared == set(_lib.EXPORTS)
    assert L.mhpc_version() >= 1


def test_info_and_cfg_parsers():
    gold = os.path.join(ROOT, "tests", "golden")
    cfg = _lib.default_config()
    _lib.check(_lib.load().mhpc_config_from_info(os.path.join(gold, "plummer.info").encode(), ctypes.byref(cfg)))
    assert cfg.integrator == 2 and cfg.theta == 0.5 and cfg.smoothing == pytest.approx(1e-4)
    assert cfg.time_step == 0.025 and cfg.sfc == 0 and cfg.gravity_force_version == 0
    assert cfg.smoothing_kernel == 1 and cfg.remove_particles == 1
    mats = (_lib.Material * 8)()
    cnt = ctypes.c_int()
    _lib.check(_lib.load().mhpc_materials_from_cfg(os.path.join(gold, "sedov.cfg").encode(), mats, 8,
                                                   ctypes.byref(cnt)))
    assert cnt.value == 1
    m = mats[0]
    assert m.interactions == 50 and m.eos_type == 9
    assert m.alpha == 1.0 and m.beta == 2.0 and m.polytropic_gamma == pytest.approx(1.6666666)
    assert m.sml == pytest.approx(0.0195)
    # malformed inputs are status codes, not crashes
    assert _lib.load().mhpc_config_from_info(b"/nonexistent.info", ctypes.byref(cfg)) == 8
    bad = os.path.join(gold, "bad_ids.cfg")
    assert _lib.load().mhpc_materials_from_cfg(bad.encode(), mats, 8, ctypes.byref(cnt)) == 8


def test_info_extension_keys(tmp_path):
    """The .info keys of this library's options (opening rule, monopole cells,
    Balsara switch, force version, precision) parse into mhpc_config, and an
    invalid opening-rule setting is a status code."""
    info = tmp_path / "ext.info"
    info.write_text("; extension keys\nintegrator 2\ntheta 0.5\nprecision 1\nthetaMixed 0.28\n"
                    "gravityMac 1\nmacAlpha 0.0018\nmacQuadAlpha 3e-4\nbalsaraSwitch true\n"
                    "gravityForceVersion 2\nsfc 1\n")
    cfg = _lib.default_config()
    _lib.check(_lib.load().mhpc_config_from_info(str(info).encode(), ctypes.byref(cfg)))
    assert cfg.precision == 1 and cfg.theta_mixed == pytest.approx(0.28)
    assert cfg.gravity_mac == 1 and cfg.mac_alpha == pytest.approx(1.8e-3)
    assert cfg.mac_quad_alpha == pytest.approx(3e-4) and cfg.balsara == 1
    assert cfg.gravity_force_version == 2 and cfg.sfc == 1
    bad = tmp_path / "bad.info"
    bad.write_text("gravityMac 1\nmacAlpha 0\n")
    assert _lib.load().mhpc_config_from_info(str(bad).encode(), ctypes.byref(_lib.default_config())) == 8


def test_generators_shapes_and_seeds():
    a = ics.plummer(1000, seed=1)
    b = ics.plummer(1000, seed=1)
    assert np.array_equal(a["x"], b["x"])
    r = np.sqrt(a["x"] ** 2 + a["y"] ** 2 + a["z"] ** 2)
    assert r.max() < 10.5
    s = ics.sedov(nside=8)
    assert len(s["x"]) == 512 and abs(s["mass"].sum() - 1.0) < 1e-12
    e_tot = (s["mass"] * s["e"]).sum()
    assert abs(e_tot - (1.0 + 1e-6)) < 1e-9
    c = ics.rotating_cloud(5000, seed=2)
    rr = np.sqrt(c["x"] ** 2 + c["y"] ** 2 + c["z"] ** 2)
    assert rr.max() <= 1.0 and abs(c["omega"] ** 2 - 0.48) < 1e-12
