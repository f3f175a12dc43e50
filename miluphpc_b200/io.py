"""Particle state files with the reference's dataset names, as .npz.

milupHPC reads its initial conditions from HDF5 (`/x`, `/v` as N x 3,
`/m`, `/materialId`, `/u`, `/rho`; src/miluphpc.cpp:157-300) and writes one
file per output step, `ts%06d.h5` (`/time`, `/x`, `/v`, `/key`, `/m`, `/proc`,
`/rho`, `/p`, `/e`, `/sml`, `/noi`, `/cs`, `/drhodt`; src/miluphpc.cpp:3451-3560).
No HDF5 library is available to this package, so the same datasets are kept
in NumPy .npz archives under the same names and shapes; a file written by an
HDF5 tool with those datasets converts one-to-one.
"""
import numpy as np

INPUT_SETS = ("x", "v", "m", "materialId", "u", "rho", "sml")


def read_initial_conditions(path):
    """State dict for Miluphpc from an .npz with the reference's input
    datasets (x and v as N x 3; m; optional materialId, u -> e, rho, sml)."""
    with np.load(path) as f:
        d = {k: f[k] for k in f.files}
    for k in ("x", "v", "m"):
        if k not in d:
            raise KeyError("initial conditions need /%s" % k)
    x = np.asarray(d["x"], dtype=np.float64).reshape(-1, 3)
    v = np.asarray(d["v"], dtype=np.float64).reshape(-1, 3)
    n = len(x)
    if len(v) != n or len(d["m"]) != n:
        raise ValueError("datasets /x, /v, /m differ in length")
    S = dict(x=x[:, 0].copy(), y=x[:, 1].copy(), z=x[:, 2].copy(),
             vx=v[:, 0].copy(), vy=v[:, 1].copy(), vz=v[:, 2].copy(),
             mass=np.asarray(d["m"], dtype=np.float64).copy())
    if "materialId" in d:
        S["material_id"] = np.asarray(d["materialId"], dtype=np.int32).copy()
    if "u" in d:
        S["e"] = np.asarray(d["u"], dtype=np.float64).copy()
    for k in ("rho", "sml"):
        if k in d:
            S[k] = np.asarray(d[k], dtype=np.float64).copy()
    return S


def output_name(step):
    """The reference's per-step file name, with the .npz suffix."""
    return "ts%06d.npz" % step


def write_output(path, sim, time):
    """One output file of the current state of a Miluphpc simulation, with
    the reference's dataset names (single rank: /proc is all zeros)."""
    n = sim.n
    keys, perm = sim.export_sorted()
    key = np.zeros(n, dtype=np.uint64)
    key[perm] = keys
    out = {"time": np.array([time], dtype=np.float64),
           "x": np.stack([sim.numpy("x"), sim.numpy("y"), sim.numpy("z")], axis=1),
           "v": np.stack([sim.numpy("vx"), sim.numpy("vy"), sim.numpy("vz")], axis=1),
           "key": key, "m": sim.numpy("mass"), "proc": np.zeros(n, dtype=np.int32)}
    if sim.cfg.sph:
        for name, field in (("rho", "rho"), ("p", "p"), ("e", "e"), ("sml", "sml"), ("cs", "cs"),
                            ("drhodt", "drhodt")):
            out[name] = sim.numpy(field)
        out["noi"] = sim.numpy("noi")
    np.savez(path, **out)
    return path
