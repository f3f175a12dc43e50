"""B200-native right-hand side of milupHPC (SFC keys, sort, octree, Barnes-Hut,
neighbour search, SPH) behind the C ABI of include/mhpc.h."""
from . import _lib  # noqa: F401
from ._lib import Config, Material, MhpcError, Particles, default_config, load  # noqa: F401


def __getattr__(name):
    # torch-backed helpers load lazily so that `import miluphpc_b200` works
    # without initialising CUDA
    if name in ("Miluphpc", "config_from_info", "materials_from_cfg", "material", "direct_gravity"):
        from . import miluphpc as _m
        return getattr(_m, name)
    raise AttributeError(name)
