"""State files with the reference's dataset names (.npz bridge for the HDF5
initial conditions and ts%06d outputs of src/miluphpc.cpp:157-300, 3451-3560)."""
import numpy as np
import pytest

from miluphpc_b200 import io as mio


def _ic(path, n=1000, seed=3):
    rng = np.random.default_rng(seed)
    d = dict(x=rng.normal(size=(n, 3)), v=rng.normal(size=(n, 3)), m=np.full(n, 1.0 / n),
             materialId=np.zeros(n, dtype=np.int32), u=rng.uniform(1, 2, n), rho=np.ones(n))
    np.savez(path, **d)
    return d


def test_read_initial_conditions(tmp_path):
    p = tmp_path / "ic.npz"
    d = _ic(p)
    S = mio.read_initial_conditions(p)
    np.testing.assert_array_equal(S["x"], d["x"][:, 0])
    np.testing.assert_array_equal(S["vz"], d["v"][:, 2])
    np.testing.assert_array_equal(S["e"], d["u"])
    assert S["material_id"].dtype == np.int32
    assert mio.output_name(7) == "ts000007.npz"
    bad = tmp_path / "bad.npz"
    np.savez(bad, x=d["x"], v=d["v"][:10], m=d["m"])
    with pytest.raises(ValueError):
        mio.read_initial_conditions(bad)


@pytest.mark.gpu
def test_write_output_roundtrip(tmp_path, cuda):
    from miluphpc_b200.miluphpc import Miluphpc
    from oracle import oracle as O
    from tests.helpers import gravity_cfg
    p = tmp_path / "ic.npz"
    _ic(p, n=4096)
    S = mio.read_initial_conditions(p)
    sim = Miluphpc(gravity_cfg(sfc=1), S)
    sim.integrate(0)
    out = mio.write_output(tmp_path / mio.output_name(1), sim, 0.025)
    f = np.load(out)
    assert f["x"].shape == (4096, 3) and f["time"][0] == 0.025
    np.testing.assert_array_equal(f["x"][:, 1], sim.numpy("y"))
    # leapfrog drifts before its right-hand side, so the written keys are the
    # Hilbert keys of the written positions
    x, y, z = f["x"][:, 0], f["x"][:, 1], f["x"][:, 2]
    assert np.array_equal(f["key"], O.keys(x, y, z, O.bbox(x, y, z), 1))
    S2 = mio.read_initial_conditions(out)
    np.testing.assert_array_equal(S2["vx"], sim.numpy("vx"))
    sim.close()
