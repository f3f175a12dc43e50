"""ctypes front end of the FP64 CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: the oracle is the checker for the CUDA product path.
Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
its reference arm) import this module; the product package never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")

_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_l = ctypes.POINTER(ctypes.c_long)
_u = ctypes.POINTER(ctypes.c_uint64)


def build(force=False):
    """Compile oracle.cpp into liboracle.so (g++, OpenMP, no FMA contraction
    so FP64 sums round like the reference's -fmad=false build)."""
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC):
        return LIB_PATH
    cmd = ["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC", "-std=c++17",
           SRC, "-o", LIB_PATH]
    subprocess.check_call(cmd)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_bbox.argtypes = [_d, _d, _d, ctypes.c_int, _d]
        L.orc_keys.argtypes = [_d, _d, _d, ctypes.c_int, _d, ctypes.c_int, _u]
        L.orc_lebesgue2hilbert.argtypes = [ctypes.c_uint64]
        L.orc_lebesgue2hilbert.restype = ctypes.c_uint64
        L.orc_sort.argtypes = [_u, ctypes.c_int, _u, _i]
        L.orc_tree_build.argtypes = [_d, _d, _d, ctypes.c_int, ctypes.c_int, _d, _i, _i, _d, _d, _d, _d]
        L.orc_tree_build.restype = ctypes.c_int
        L.orc_com.argtypes = [_i, _i, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _d, _d, _d]
        L.orc_tree_nodeset.argtypes = [_i, ctypes.c_int, _u, _i, ctypes.c_int]
        L.orc_tree_nodeset.restype = ctypes.c_int
        L.orc_gravity_v2.argtypes = [_d, _d, _d, _d, _i, _i, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, _d, _d, _d]
        L.orc_gravity_v2_sample.argtypes = [_d, _d, _d, _d, _i, _i, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, _d, _d, _d, ctypes.c_int]
        L.orc_gravity_v1.argtypes = [_d, _d, _d, _d, _i, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, _d, _d, _d, _i]
        L.orc_direct.argtypes = [_d, _d, _d, _d, ctypes.c_int, _i, ctypes.c_int, ctypes.c_double,
                                 _d, _d, _d, _d]
        L.orc_frnn.argtypes = [_d, _d, _d, _d, ctypes.c_int, _l, _i]
        L.orc_density.argtypes = [_d, _d, _d, _d, _d, ctypes.c_int, _l, _i, ctypes.c_int, ctypes.c_int, _d]
        L.orc_eos.argtypes = [ctypes.c_int, ctypes.c_int, _d, _d, _d, _d, _d]
        L.orc_forces.argtypes = [_d] * 11 + [ctypes.c_int, _l, _i, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_d] * 7
        L.orc_balsara.argtypes = [_d] * 10 + [ctypes.c_int, _l, _i, ctypes.c_int, ctypes.c_int, _d, _d, _d]
        L.orc_variable_h.argtypes = [_d, _d, _d, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _i, ctypes.c_double]
        L.orc_variable_h.restype = ctypes.c_int
        L.orc_band_fixup.argtypes = [_d, _d, _d, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double]
        L.orc_band_fixup.restype = ctypes.c_int
        L.orc_euler.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int] + [_d] * 18
        L.orc_leapfrog_x.argtypes = [ctypes.c_int, ctypes.c_double] + [_d] * 12
        L.orc_leapfrog_v.argtypes = [ctypes.c_int, ctypes.c_double] + [_d] * 9
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_quad.argtypes = [_i, _i, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _d, _d, _d, _d]
        L.orc_cell_bmax2.argtypes = [_i, _i, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _d, _d, _d]
        L.orc_gravity_group_crit.argtypes = [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             _d, _d, _d, _i, _d]
        L.orc_gravity_group.argtypes = [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        _d, _d, _d, _i]
        L.orc_gravity_boxes.argtypes = [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, _d, ctypes.c_double,
                                        _d, _d, _d, _i, _i]
        L.orc_gravity_boxes_rel.argtypes = [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _d,
                                            ctypes.c_double, _d, ctypes.c_double, ctypes.c_int, _d, _d, _d, _i, _i]
        L.orc_gravity_boxes_mono.argtypes = [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _d,
                                             ctypes.c_double, ctypes.c_double, _d, _d, _d, _i, _i]
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def num_threads():
    return lib().orc_num_threads()


def bbox(x, y, z):
    out = np.zeros(6)
    x, y, z = _f64(x), _f64(y), _f64(z)
    lib().orc_bbox(_p(x), _p(y), _p(z), len(x), _p(out))
    return out


def keys(x, y, z, bb, curve=0):
    x, y, z = _f64(x), _f64(y), _f64(z)
    bb = _f64(bb)
    out = np.zeros(len(x), dtype=np.uint64)
    lib().orc_keys(_p(x), _p(y), _p(z), len(x), _p(bb), int(curve), _p(out, _u))
    return out


def lebesgue2hilbert(k):
    return int(lib().orc_lebesgue2hilbert(ctypes.c_uint64(int(k))))


def sort(k):
    k = np.ascontiguousarray(k, dtype=np.uint64)
    ks = np.zeros_like(k)
    perm = np.zeros(len(k), dtype=np.int32)
    lib().orc_sort(_p(k, _u), len(k), _p(ks, _u), _p(perm, _i))
    return ks, perm


class Tree:
    """Reference-layout octree (child[8*num_nodes], cells from n upward)."""

    def __init__(self, x, y, z, m, bb, num_nodes=None, com=True, com_max_level=21):
        n = len(x)
        self.n = n
        self.num_nodes = num_nodes or (2 * n + 20000)
        nn = self.num_nodes
        self.child = np.zeros(8 * nn, dtype=np.int32)
        self.level = np.zeros(nn, dtype=np.int32)
        self.x = np.zeros(nn); self.y = np.zeros(nn); self.z = np.zeros(nn); self.m = np.zeros(nn)
        self.x[:n] = x; self.y[:n] = y; self.z[:n] = z; self.m[:n] = m
        px, py, pz = _f64(x), _f64(y), _f64(z)
        bb = _f64(bb)
        r = lib().orc_tree_build(_p(px), _p(py), _p(pz), n, nn, _p(bb), _p(self.child, _i),
                                 _p(self.level, _i), _p(self.x), _p(self.y), _p(self.z), _p(self.m))
        if r < 0:
            raise RuntimeError("oracle tree build failed: %d" % r)
        self.nodes = r
        if com:
            lib().orc_com(_p(self.child, _i), _p(self.level, _i), n, r, int(com_max_level),
                          _p(self.x), _p(self.y), _p(self.z), _p(self.m))

    def nodeset(self):
        cap = self.nodes - self.n + 8
        pre = np.zeros(cap, dtype=np.uint64)
        lev = np.zeros(cap, dtype=np.int32)
        c = lib().orc_tree_nodeset(_p(self.child, _i), self.n, _p(pre, _u), _p(lev, _i), cap)
        return pre[:c], lev[:c]


def gravity_v2(tree, sorted_perm, radius, theta, eps2):
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    lib().orc_gravity_v2(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(tree.child, _i),
                         _p(sp, _i), n, float(radius), float(theta), float(eps2),
                         _p(ax), _p(ay), _p(az))
    return ax, ay, az


def gravity_v2_sample(tree, sorted_perm, radius, theta, eps2, stride):
    """v2 walk for every stride-th warp group only (timing sample)."""
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    lib().orc_gravity_v2_sample(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(tree.child, _i),
                                _p(sp, _i), n, float(radius), float(theta), float(eps2),
                                _p(ax), _p(ay), _p(az), int(stride))
    return ax, ay, az


def gravity_v1(tree, radius, theta, eps2):
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    lib().orc_gravity_v1(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(tree.child, _i), n,
                         float(radius), float(theta), float(eps2), _p(ax), _p(ay), _p(az),
                         _p(cnt, _i))
    return ax, ay, az, cnt


def direct(x, y, z, m, targets, eps2):
    x, y, z, m = _f64(x), _f64(y), _f64(z), _f64(m)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    nt = len(t)
    ax = np.zeros(nt); ay = np.zeros(nt); az = np.zeros(nt); pot = np.zeros(nt)
    lib().orc_direct(_p(x), _p(y), _p(z), _p(m), len(x), _p(t, _i), nt, float(eps2),
                     _p(ax), _p(ay), _p(az), _p(pot))
    return ax, ay, az, pot


def frnn(x, y, z, h):
    x, y, z, h = _f64(x), _f64(y), _f64(z), _f64(h)
    n = len(x)
    off = np.zeros(n + 1, dtype=np.int64)
    lib().orc_frnn(_p(x), _p(y), _p(z), _p(h), n, _p(off, _l), None)
    nbr = np.zeros(int(off[-1]), dtype=np.int32)
    lib().orc_frnn(_p(x), _p(y), _p(z), _p(h), n, _p(off, _l), _p(nbr, _i))
    return off, nbr


def density(x, y, z, m, h, off, nbr, avg_h=False, kernel=1):
    """kernel: 0 spiky, 1 cubic spline, 2/3/4 Wendland C2/C4/C6."""
    x, y, z, m, h = _f64(x), _f64(y), _f64(z), _f64(m), _f64(h)
    rho = np.zeros(len(x))
    lib().orc_density(_p(x), _p(y), _p(z), _p(m), _p(h), len(x), _p(off, _l), _p(nbr, _i),
                      int(avg_h), int(kernel), _p(rho))
    return rho


def eos(eos_type, par, rho, e, p_prev, si_units=False):
    """par = (K, gamma, rho_0, bulk_modulus, n); the Murnaghan and isothermal
    sound speeds are the constants of initializeSoundSpeed."""
    n = len(rho)
    par = np.concatenate([_f64(par)[:5], np.zeros(max(0, 5 - len(par))), [1.0 if si_units else 0.0]])
    rho, e = _f64(rho), _f64(e)
    p = np.array(p_prev, dtype=np.float64, copy=True)
    cs = np.zeros(n)
    lib().orc_eos(n, int(eos_type), _p(par), _p(rho), _p(e), _p(p), _p(cs))
    return p, cs


def forces(x, y, z, vx, vy, vz, m, h, rho, p, cs, off, nbr, alpha, beta, avg_h=False,
           integrate_energy=True, integrate_sml=False, bal=None, kernel=1):
    arrs = [_f64(a) for a in (x, y, z, vx, vy, vz, m, h, rho, p, cs)]
    n = len(x)
    outs = [np.zeros(n) for _ in range(6)]
    b = _f64(bal) if bal is not None else None
    lib().orc_forces(*[_p(a) for a in arrs], n, _p(off, _l), _p(nbr, _i), float(alpha),
                     float(beta), int(avg_h), int(integrate_energy), int(integrate_sml), int(kernel),
                     *[_p(o) for o in outs], _p(b) if b is not None else None)
    return outs


def balsara(x, y, z, vx, vy, vz, m, h, rho, cs, off, nbr, avg_h=False, kernel=1):
    """Balsara switch: (div v, curl v [n x 3], f)."""
    arrs = [_f64(a) for a in (x, y, z, vx, vy, vz, m, h, rho, cs)]
    n = len(x)
    divv, curl, f = np.zeros(n), np.zeros((n, 3)), np.zeros(n)
    lib().orc_balsara(*[_p(a) for a in arrs], n, _p(off, _l), _p(nbr, _i), int(avg_h), int(kernel), _p(divv),
                      _p(curl), _p(f))
    return divv, curl, f


def euler(st, dt, gravity=True, sph=True, integrate_density=False, integrate_energy=False,
          integrate_sml=False):
    """ExplicitEulerNS::Kernel::update on a dict of float64 arrays (copied)."""
    out = {k: np.array(v, dtype=np.float64, copy=True) for k, v in st.items()}
    n = len(out["x"])
    z = np.zeros(n)
    names = ["x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay", "g_az", "rho", "drhodt", "e",
             "dedt", "sml", "dsmldt"]
    for k in names:
        out.setdefault(k, z.copy())
    lib().orc_euler(n, float(dt), int(gravity), int(sph), int(integrate_density), int(integrate_energy),
                    int(integrate_sml), *[_p(out[k]) for k in names])
    return out


def variable_h(x, y, z, h, target, tol=5, max_nb=180, max_iter=5):
    x, y, z = _f64(x), _f64(y), _f64(z)
    h = np.array(h, dtype=np.float64, copy=True)
    cnt = np.zeros(len(x), dtype=np.int32)
    sweeps = lib().orc_variable_h(_p(x), _p(y), _p(z), _p(h), len(x), int(target), int(tol),
                                  int(max_nb), int(max_iter), _p(cnt, _i), _box_edge(x, y, z))
    return h, cnt, sweeps


def band_fixup(x, y, z, h, target, tol=5, rounds=8):
    """Neighbour-band repair rounds on h (returns (h, out-of-band count before
    the first round))."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    h = np.array(h, dtype=np.float64, copy=True)
    before = lib().orc_band_fixup(_p(x), _p(y), _p(z), _p(h), len(x), int(target), int(tol), int(rounds),
                                  _box_edge(x, y, z))
    return h, before


def _box_edge(x, y, z):
    bb = bbox(x, y, z)
    return float(bb[1] - bb[0])


def quad(tree, max_level=21):
    q = np.zeros(6 * tree.num_nodes)
    lib().orc_quad(_p(tree.child, _i), _p(tree.level, _i), tree.n, tree.nodes, int(max_level),
                   _p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(q))
    return q


def gravity_group(tree, sorted_perm, radius, theta, eps2, q=None, gsize=32):
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    lib().orc_gravity_group(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m),
                            _p(q) if q is not None else None, _p(tree.child, _i),
                            _p(tree.level, _i), _p(sp, _i), n, int(gsize), float(radius),
                            float(theta), float(eps2), _p(ax), _p(ay), _p(az), _p(cnt, _i))
    return ax, ay, az, cnt


def cell_bmax2(tree, max_level=21):
    b = np.zeros(tree.num_nodes)
    lib().orc_cell_bmax2(_p(tree.child, _i), _p(tree.level, _i), tree.n, tree.nodes, int(max_level),
                         _p(tree.x), _p(tree.y), _p(tree.z), _p(b))
    return b


def gravity_group_crit(tree, sorted_perm, crit, eps2, q=None, gsize=32):
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    crit = np.ascontiguousarray(crit, dtype=np.float64)
    lib().orc_gravity_group_crit(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m),
                                 _p(q) if q is not None else None, _p(tree.child, _i),
                                 _p(tree.level, _i), _p(sp, _i), n, int(gsize), 1.0, 1.0, float(eps2),
                                 _p(ax), _p(ay), _p(az), _p(cnt, _i), _p(crit))
    return ax, ay, az, cnt


def gravity_boxes(tree, sorted_perm, radius, theta, eps2, q, gsize=64, nsub=8, h=None, h_factor=0.0):
    """Interaction-list walk of the mixed path in FP64 (sub-box criterion)."""
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    nq = np.zeros(n, dtype=np.int32)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    hh = _f64(h) if h is not None else None
    lib().orc_gravity_boxes(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(q), _p(tree.child, _i),
                            _p(tree.level, _i), _p(sp, _i), n, int(gsize), int(nsub), float(radius),
                            float(theta), float(eps2), _p(hh) if hh is not None else None, float(h_factor),
                            _p(ax), _p(ay), _p(az), _p(cnt, _i), _p(nq, _i))
    return ax, ay, az, cnt, nq


def gravity_boxes_rel(tree, sorted_perm, radius, theta, eps2, q, amag, alpha, lpow=3, gsize=64, nsub=8):
    """Sub-box walk with the relative opening criterion added (FP64)."""
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    nq = np.zeros(n, dtype=np.int32)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    am = _f64(amag)
    lib().orc_gravity_boxes_rel(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(q), _p(tree.child, _i),
                                _p(tree.level, _i), _p(sp, _i), n, int(gsize), int(nsub), float(radius),
                                float(theta), float(eps2), None, 0.0, _p(am), float(alpha), int(lpow),
                                _p(ax), _p(ay), _p(az), _p(cnt, _i), _p(nq, _i))
    return ax, ay, az, cnt, nq


def gravity_boxes_mono(tree, sorted_perm, radius, theta, eps2, q, amag, alpha, mono_alpha, gsize=64, nsub=8):
    """Relative-rule walk where accepted cells whose quadrupole term is below
    mono_alpha |a| enter as monopoles (FP64); returns ax, ay, az, nodes,
    cells with quadrupole (per particle)."""
    n = tree.n
    ax = np.zeros(n); ay = np.zeros(n); az = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32); nq = np.zeros(n, dtype=np.int32)
    sp = np.ascontiguousarray(sorted_perm, dtype=np.int32)
    lib().orc_gravity_boxes_mono(_p(tree.x), _p(tree.y), _p(tree.z), _p(tree.m), _p(q), _p(tree.child, _i),
                                 _p(tree.level, _i), _p(sp, _i), n, int(gsize), int(nsub), float(radius),
                                 float(theta), float(eps2), _p(_f64(amag)), float(alpha), float(mono_alpha),
                                 _p(ax), _p(ay), _p(az), _p(cnt, _i), _p(nq, _i))
    return ax, ay, az, cnt, nq
