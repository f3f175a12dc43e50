"""Time milupHPC's own single-rank gravity kernels on a B200 (test
infrastructure: the reference harness oracle/_ref/ref_gravity, built from the
reference sources by build_ref.py).

Workload: the 131,072-particle Plummer sphere of the single-rank reference
case (seed 1 of miluphpc_b200.ics.plummer, Lebesgue keys, theta 0.5,
eps^2 = 1e-4).  Before the harness sees the input, the CPU checks that the
reference kernels stay in bounds on it (distinct 21-level keys, tree depth
<= 16, node pool, n a multiple of 65536 for the strided per-particle loops);
a failed check stops here without running anything on the GPU.  The
harness runs one right-hand side untimed, then `repeats` timed ones, and
prints the mean milliseconds per stage; the accelerations of its first pass
are compared with the oracle's emulation of computeForces_v2.

    python oracle/ref_harness/time_ref.py OUT.json [repeats]
    python oracle/ref_harness/time_ref.py OUT.json [repeats] --sph   (fixed-h SPH, 64^3 Sedov)
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from make_golden import MAX_DEPTH_V2, check_tree, header  # noqa: E402
from miluphpc_b200 import ics  # noqa: E402
from oracle import oracle as O  # noqa: E402

N, SEED, THETA, EPS2 = 131072, 1, 0.5, 1e-4


def main():
    out_json = sys.argv[1]
    repeats = int(sys.argv[2]) if len(sys.argv) > 2 else 10
    S = ics.plummer(N, seed=SEED)
    x, y, z, m = S["x"], S["y"], S["z"], S["mass"]
    bb = O.bbox(x, y, z)
    if N % 65536 != 0:
        raise SystemExit("n must be a multiple of 65536 above 65536")
    _, depth = check_tree(x, y, z, m, bb, MAX_DEPTH_V2)
    keys = O.keys(x, y, z, bb, 0)
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gravity")
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            f.write(header(N, THETA, EPS2, []))
            for a in (x, y, z, m):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(keys, dtype="<u8").tobytes())
        res = subprocess.run([exe, fin, fout, str(repeats)], check=True, capture_output=True, text=True)
        raw = open(fout, "rb").read()
    times = {}
    for line in res.stdout.splitlines():
        f = line.split()
        if len(f) == 3 and f[0] == "time_ms":
            times[f[1]] = float(f[2])
    # the reference's accelerations (last 3 n doubles of the output) against
    # the oracle's emulation of its walk on the same tree
    g = np.frombuffer(raw[-24 * N:], dtype="<f8").reshape(3, N)
    _, perm = O.sort(keys)
    T = O.Tree(x, y, z, m, bb)
    ox, oy, oz = O.gravity_v2(T, perm, 0.5 * (bb[1] - bb[0]), THETA, EPS2)
    num = np.sqrt((g[0] - ox) ** 2 + (g[1] - oy) ** 2 + (g[2] - oz) ** 2)
    rel = num / np.sqrt(ox ** 2 + oy ** 2 + oz ** 2)
    out = {"workload": "plummer131k: N = 131072 Plummer (seed %d), Lebesgue, theta %g, eps2 %g" % (SEED, THETA, EPS2),
           "tree_depth": depth, "repeats": repeats, "ms_per_rhs_by_stage": times,
           "particle_rhs_per_s": N / (times["total"] / 1e3),
           "max_rel_diff_vs_oracle_v2": float(rel.max()),
           "stages": "resetArrays + computeBoundingBox, buildTree, calculateCentersOfMass (21 levels), "
                     "prepareSorting + sortArray (CUB), computeForces_v2; each launch wrapper synchronises",
           "keys": "not timed (getParticleKeys is not run by the harness; the oracle's keys are sorted)"}
    with open(out_json, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


def main_sph():
    """The reference's fixed-h SPH right-hand side on the 64^3 Sedov lattice
    (seed 2 of miluphpc_b200.ics.sedov, the bench workload sedov262k; ideal
    gas gamma 5/3, alpha 1, beta 2, cubic spline), after the CPU checks of
    the SPH fixtures: distinct keys, the node pool, fewer than 150 neighbours
    per particle (fixedRadiusNN v0 stores without a bound check), positive
    masses and energies.  Its density is compared with the oracle's."""
    out_json = sys.argv[1]
    repeats = int(sys.argv[2]) if len(sys.argv) > 2 and not sys.argv[2].startswith("-") else 10
    from make_golden import MAXNB_MARGIN, check_tree as ct
    S = ics.sedov(nside=64, seed=2)
    n = len(S["x"])
    x, y, z, m = S["x"], S["y"], S["z"], S["mass"]
    bb = O.bbox(x, y, z)
    if n % 65536 != 0 or n > (1 << 20):
        raise SystemExit("n must be a multiple of 65536 up to 2^20")
    _, depth = ct(x, y, z, m, bb, 21)
    off, nbr = O.frnn(x, y, z, S["sml"])
    noi = np.diff(off)
    if noi.max() > MAXNB_MARGIN or (m <= 0).any() or (S["e"] < 0).any():
        raise SystemExit("sph input outside the checked range")
    zeros = np.zeros(n)
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_sph")
    par = [60, 1.0, 2.0, 9, 0.0, 5.0 / 3.0]
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            f.write(header(n, 0.0, 0.0, par))
            for a in (x, y, z, m, S["vx"], S["vy"], S["vz"], S["sml"], S["e"], zeros, zeros):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        res = subprocess.run([exe, fin, fout, str(repeats)], check=True, capture_output=True, text=True)
        raw = open(fout, "rb").read()
    times = {}
    for line in res.stdout.splitlines():
        f = line.split()
        if len(f) == 3 and f[0] == "time_ms":
            times[f[1]] = float(f[2])
    # rho follows noi[n] and nnl[maxnb n] after the 56-byte header
    maxnb = int(np.frombuffer(raw[52:56], dtype="<i4")[0])
    pos = 56 + 4 * n + 4 * maxnb * n
    rho = np.frombuffer(raw[pos:pos + 8 * n], dtype="<f8")
    rho_o = O.density(x, y, z, m, S["sml"], off, nbr)
    out = {"workload": "sedov262k: 64^3 jittered lattice (seed 2), fixed h = 2.5 dx, ideal gas, cubic spline",
           "tree_depth": depth, "neighbours": [int(noi.min()), int(noi.max())], "repeats": repeats,
           "ms_per_rhs_by_stage": times, "particle_rhs_per_s": n / (times["total"] / 1e3),
           "max_rel_diff_rho_vs_oracle": float(np.max(np.abs(rho - rho_o) / rho_o)),
           "stages": "resetArrays + noi/nnl memsets + computeBoundingBox, buildTree, fixedRadiusNN, "
                     "calculateDensity, calculateSoundSpeed + calculatePressure, internalForces; each launch "
                     "wrapper synchronises"}
    with open(out_json, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    if "--sph" in sys.argv:
        sys.argv.remove("--sph")
        main_sph()
    else:
        main()
