"""Generate the reference fixtures ref_gravity_*.npz, ref_sph*.npz,
ref_hilbert.npz (CPU only) and ref_integrators.npz.

The fixtures hold seeded inputs together with the outputs of milupHPC's own
kernels, run by the reference harness (oracle/_ref/ref_gravity and
oracle/_ref/ref_sph, built from the reference sources by
oracle/ref_harness/build_ref.py) on a GPU.  tests/test_ref_golden.py checks
the oracle and the CUDA path against them.

Every input is checked on the CPU with the oracle before the harness sees it,
so that the reference kernels only run on inputs they handle in bounds:
distinct 21-level keys (buildTree subdivides until two particles separate),
tree depth <= 16 (computeForces_v2 keeps 128 stack entries per warp, one
level adds at most 7), node pool large enough, fewer neighbours than
MAX_NUM_INTERACTIONS (fixedRadiusNN v0 stores without a bound check),
positive masses, pressures and energies.

    python tests/golden/make_golden.py [--out DIR] [--check-only]
"""
import argparse
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from miluphpc_b200 import ics  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
MAX_DEPTH_V2 = 16
MAXNB_MARGIN = 150

GRAVITY_CASES = [
    # name, n, seed, curve (0 Lebesgue, 1 Hilbert), theta, eps2
    ("ref_gravity_lebesgue", 2048, 11, 0, 0.5, 1e-4),
    ("ref_gravity_hilbert", 2048, 12, 1, 0.7, 1e-6),
]
SPH_PARAMS = dict(interactions=50, alpha=1.0, beta=2.0, eos=9, K=0.0, gamma=5.0 / 3.0)


def header(n, theta, eps2, par):
    par = list(par) + [0.0] * (8 - len(par))
    return struct.pack("<ii", n, 0) + struct.pack("<10d", theta, eps2, *par)


def walk_ref_tree(child, n, x, y, z, m):
    """Cells of the reference tree by path from the root (child slots 0..7):
    prefix (octal digits), level, centre of mass; and each particle's path."""
    cells = []
    leaf_prefix = np.full(n, -1, dtype=np.int64)
    leaf_level = np.full(n, -1, dtype=np.int32)
    stack = [(0, 0, 0)]
    while stack:
        node, prefix, level = stack.pop()
        if level > 0:
            cells.append((prefix, level, x[node], y[node], z[node], m[node]))
        for c in range(8):
            ch = int(child[8 * node + c])
            if ch < 0:
                continue
            if ch < n:
                if leaf_level[ch] >= 0:
                    raise RuntimeError("particle %d reached twice" % ch)
                leaf_prefix[ch] = (prefix << 3) | c
                leaf_level[ch] = level + 1
            else:
                stack.append((ch, (prefix << 3) | c, level + 1))
    if (leaf_level < 0).any():
        raise RuntimeError("particles missing from the reference tree")
    cells.sort()
    c = np.array(cells, dtype=object)
    return (np.array(c[:, 0], dtype=np.uint64), np.array(c[:, 1], dtype=np.int32),
            np.array(c[:, 2:6], dtype=np.float64), leaf_prefix.astype(np.uint64), leaf_level)


def check_tree(x, y, z, m, bb, max_depth):
    keys = O.keys(x, y, z, bb, 0)
    if len(np.unique(keys)) != len(keys):
        raise RuntimeError("coincident 21-level keys")
    n = len(x)
    t = O.Tree(x, y, z, m, bb)
    _, lev = t.nodeset()
    if t.nodes >= 2 * n + 20000:
        raise RuntimeError("node pool")
    if lev.max() > max_depth:
        raise RuntimeError("tree depth %d > %d" % (lev.max(), max_depth))
    return t, int(lev.max())


def gravity_case(name, n, seed, curve, theta, eps2, out, run):
    S = ics.plummer(n, seed=seed)
    x, y, z, m = S["x"], S["y"], S["z"], S["mass"]
    bb = O.bbox(x, y, z)
    _, depth = check_tree(x, y, z, m, bb, MAX_DEPTH_V2)
    keys = O.keys(x, y, z, bb, curve)
    print("%s: n=%d depth=%d" % (name, n, depth), flush=True)
    if not run:
        return
    fin = os.path.join(out, name + ".in")
    fout = os.path.join(out, name + ".out")
    with open(fin, "wb") as f:
        f.write(header(n, theta, eps2, []))
        for a in (x, y, z, m):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(keys, dtype="<u8").tobytes())
    subprocess.check_call([os.path.join(REF, "ref_gravity"), fin, fout])
    nn = 2 * n + 20000
    buf = open(fout, "rb").read()
    off = 0

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(buf, dtype=dt, count=cnt, offset=off)
        off += a.nbytes
        return a.copy()

    bbox = take("<f8", 6)
    index, _maxnb = take("<i4", 2)
    sorted_ = take("<i4", n)
    child = take("<i4", 8 * nn)
    _level = take("<i4", nn)
    nx, ny, nz, nm = (take("<f8", nn) for _ in range(4))
    ax, ay, az = (take("<f8", n) for _ in range(3))
    cp, cl, com, lp, ll = walk_ref_tree(child, n, nx, ny, nz, nm)
    np.savez_compressed(os.path.join(out, name + ".npz"), x=x, y=y, z=z, m=m, theta=theta, eps2=eps2,
                        curve=curve, bbox=bbox, cells=int(index) - n, sorted=sorted_, cell_prefix=cp,
                        cell_level=cl, cell_com=com, leaf_prefix=lp, leaf_level=ll, ax=ax, ay=ay, az=az)
    os.remove(fin)
    os.remove(fout)


def sph_input(seed=21):
    """Jittered 16x16x8 lattice of unit density with a hot centre (a small
    Sedov-like set-up), per-particle smoothing lengths within +-10 % and
    random plus radial velocities so that the viscosity term is active."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / 16
    ix, iy, iz = np.meshgrid(np.arange(16), np.arange(16), np.arange(8), indexing="ij")
    pos = [((a.ravel() + 0.5) * dx - c) for a, c in ((ix, 0.5), (iy, 0.5), (iz, 0.25))]
    pos = [p + rng.uniform(-0.1, 0.1, p.size) * dx for p in pos]
    x, y, z = pos
    n = x.size
    m = np.full(n, dx ** 3)
    h = 2.2 * dx * (1.0 + rng.uniform(-0.1, 0.1, n))
    r = np.sqrt(x * x + y * y + z * z)
    e = np.full(n, 1e-5)
    e[r < 2.0 * dx] = 10.0
    vx, vy, vz = (rng.normal(0.0, 0.01, n) for _ in range(3))
    hot = r < 3.0 * dx
    for v, c in ((vx, x), (vy, y), (vz, z)):
        v[hot] += 0.5 * c[hot] / np.maximum(r[hot], 1e-12)
    gamma = SPH_PARAMS["gamma"]
    p = (gamma - 1.0) * 1.0 * e
    cs = np.sqrt(gamma * p / 1.0)
    return dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz, sml=h, e=e, p=p, cs=cs)


def sph_case(out, run, balsara=False):
    """ref_sph: the Sedov build; ref_sph_balsara: the same with the Balsara
    switch on (harness build ref_sph_bal), which adds div v and curl v."""
    name = "ref_sph_balsara" if balsara else "ref_sph"
    S = sph_input()
    n = len(S["x"])
    bb = O.bbox(S["x"], S["y"], S["z"])
    _, depth = check_tree(S["x"], S["y"], S["z"], S["m"], bb, 21)
    off, _ = O.frnn(S["x"], S["y"], S["z"], S["sml"])
    noi = np.diff(off)
    if noi.max() > MAXNB_MARGIN or (S["m"] <= 0).any() or (S["p"] < 0).any() or (S["e"] < 0).any():
        raise RuntimeError("sph input outside the checked range")
    print("%s: n=%d depth=%d noi %d..%d" % (name, n, depth, noi.min(), noi.max()), flush=True)
    if not run:
        return
    P = SPH_PARAMS
    fin = os.path.join(out, name + ".in")
    fout = os.path.join(out, name + ".out")
    with open(fin, "wb") as f:
        f.write(header(n, 0.0, 0.0, [P["interactions"], P["alpha"], P["beta"], P["eos"], P["K"], P["gamma"]]))
        for k in ("x", "y", "z", "m", "vx", "vy", "vz", "sml", "e", "p", "cs"):
            f.write(np.ascontiguousarray(S[k], dtype="<f8").tobytes())
    subprocess.check_call([os.path.join(REF, "ref_sph_bal" if balsara else "ref_sph"), fin, fout])
    buf = open(fout, "rb").read()
    pos = 0

    def take(dt, cnt):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=cnt, offset=pos)
        pos += a.nbytes
        return a.copy()

    bbox = take("<f8", 6)
    _index, maxnb = take("<i4", 2)
    rnoi = take("<i4", n)
    nnl = take("<i4", int(maxnb) * n).reshape(n, int(maxnb))
    rho, cs, p, ax, ay, az, drhodt, dedt, dsmldt = (take("<f8", n) for _ in range(9))
    diam = take("<f8", 1)[0]
    extra = {}
    if balsara:
        extra["divv"] = take("<f8", n)
        extra["curlv"] = take("<f8", 3 * n).reshape(n, 3)
    nb_sum = np.zeros(n, dtype=np.int64)
    nb_sq = np.zeros(n, dtype=np.int64)
    for i in range(n):
        row = nnl[i, :rnoi[i]].astype(np.int64)
        if len(np.unique(row)) != len(row) or (row < 0).any() or (row >= n).any() or (row == i).any():
            raise RuntimeError("reference neighbour list of %d malformed" % i)
        nb_sum[i] = row.sum()
        nb_sq[i] = (row * row).sum()
    np.savez_compressed(os.path.join(out, name + ".npz"), **S, alpha=P["alpha"], beta=P["beta"],
                        gamma=P["gamma"], bbox=bbox, diam=diam, noi=rnoi, nb_sum=nb_sum, nb_sq=nb_sq,
                        rho=rho, cs_out=cs, p_out=p, ax=ax, ay=ay, az=az, drhodt=drhodt, dedt=dedt,
                        dsmldt=dsmldt, **extra)
    os.remove(fin)
    os.remove(fout)


def hilbert_case(out, seed=31):
    """Lebesgue -> Hilbert keys by the reference's own host-callable
    KeyNS::lebesgue2hilbert (run on the CPU, no GPU): seeded random 63-bit
    keys, the Lebesgue keys of a seeded Plummer sphere (whose positions are
    stored, so that the GPU keys can be checked too) and edge keys."""
    rng = np.random.default_rng(seed)
    rand = rng.integers(0, 1 << 63, 4096, dtype=np.uint64)
    P = ics.plummer(4096, seed=seed)
    bb = O.bbox(P["x"], P["y"], P["z"])
    pk = O.keys(P["x"], P["y"], P["z"], bb, 0)
    edge = np.array([0, 1, 7, 8, (1 << 63) - 1, (1 << 60), (1 << 62) + 5, 0o1234567012345670123456],
                    dtype=np.uint64)
    leb = np.concatenate([rand, pk, edge])
    fin = os.path.join(out, "ref_hilbert.in")
    fout = os.path.join(out, "ref_hilbert.out")
    with open(fin, "wb") as f:
        f.write(struct.pack("<i", len(leb)))
        f.write(np.ascontiguousarray(leb, dtype="<u8").tobytes())
    subprocess.check_call([os.path.join(REF, "ref_gravity"), "--hilbert", fin, fout])
    hil = np.frombuffer(open(fout, "rb").read(), dtype="<u8").copy()
    np.savez_compressed(os.path.join(out, "ref_hilbert.npz"), lebesgue=leb, hilbert=hil, x=P["x"], y=P["y"],
                        z=P["z"], n_random=len(rand), n_plummer=len(pk))
    os.remove(fin)
    os.remove(fout)


INTEG_FIELDS = ["x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "g_ax", "g_ay", "g_az", "rho", "drhodt", "e",
                "dedt", "sml", "dsmldt", "p", "cs", "gx2", "gy2", "gz2", "pax", "pay", "paz"]
INTEG_OUT = [("euler", ["x", "y", "z", "vx", "vy", "vz", "e", "sml"]),
             ("leapfrog", ["x", "y", "z", "g_ax_old", "g_ay_old", "g_az_old", "vx", "vy", "vz"]),
             ("predictor", ["x", "y", "z", "vx", "vy", "vz", "e", "sml", "cs", "p"]),
             ("corrector", ["x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "e", "dedt", "sml", "dsmldt"])]


def integrators_case(out, n=4096, seed=41, dt=3.7e-3):
    """The reference's integrator update kernels (ref_integrators, Sedov
    parameter.h: INTEGRATE_ENERGY, INTEGRATE_SML) on a seeded random state:
    positive e, sml, rho, p, c_s; some dedt negative enough to hit the
    energy floors (1e-50 in Euler, 1e-6 in the predictor-corrector)."""
    rng = np.random.default_rng(seed)
    st = {k: rng.normal(0.0, 1.0, n) for k in INTEG_FIELDS}
    for k in ("rho", "e", "sml", "p", "cs"):
        st[k] = np.abs(st[k]) + 0.1
    st["dedt"][:64] = -1e6
    if not all(np.isfinite(v).all() for v in st.values()):
        raise RuntimeError("non-finite input")
    fin = os.path.join(out, "ref_integrators.in")
    fout = os.path.join(out, "ref_integrators.out")
    with open(fin, "wb") as f:
        f.write(struct.pack("<id", n, dt))
        for k in INTEG_FIELDS:
            f.write(np.ascontiguousarray(st[k], dtype="<f8").tobytes())
    subprocess.check_call([os.path.join(REF, "ref_integrators"), fin, fout])
    raw = np.frombuffer(open(fout, "rb").read(), dtype="<f8")
    res, pos = {}, 0
    for stage, names in INTEG_OUT:
        for k in names:
            res[stage + "_" + k] = raw[pos:pos + n].copy()
            pos += n
    np.savez_compressed(os.path.join(out, "ref_integrators.npz"), dt=dt, **{"in_" + k: v for k, v in st.items()},
                        **res)
    os.remove(fin)
    os.remove(fout)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--check-only", action="store_true", help="run the CPU input checks only")
    ap.add_argument("--only", default=None, help="comma-separated fixture names to make")
    a = ap.parse_args()
    only = a.only.split(",") if a.only else None
    os.makedirs(a.out, exist_ok=True)
    O.build()
    for case in GRAVITY_CASES:
        if only is None or case[0] in only:
            gravity_case(*case, out=a.out, run=not a.check_only)
    if only is None or "ref_sph" in only:
        sph_case(a.out, run=not a.check_only)
    if only is None or "ref_sph_balsara" in only:
        sph_case(a.out, run=not a.check_only, balsara=True)
    if (only is None or "ref_hilbert" in only) and not a.check_only:
        hilbert_case(a.out)
    if (only is None or "ref_integrators" in only) and not a.check_only:
        integrators_case(a.out)


if __name__ == "__main__":
    main()
