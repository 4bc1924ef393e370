"""dwg_b200 -- B200-native (sm_100a) DWG reconstruction hot path.

The compute lives in ``libdwg_b200.so`` (hand-written CUDA behind the C ABI of
``include/dwg_b200.h``); this package is the host-side mirror of the
reference's operator classes (``turbo``), the ctypes binding (``capi``), the
build step (``build``) and seeded synthetic workloads (``datasets``).
"""
from . import capi  # noqa: F401

__all__ = ["capi", "turbo", "datasets", "build"]


def __getattr__(name):
    if name in ("turbo", "datasets", "build", "learned"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
