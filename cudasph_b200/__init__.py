"""cudasph_b200 -- CUDAsph's per-step SPH + self-gravity pipeline on B200 (sm_100a).

The compute path is the C ABI of ``_lib/libcudasph_b200.so`` (declared in
``include/cudasph_b200.h``); this package holds the CUDA sources
(``csrc/``), their in-tree build (``build.py``), the ctypes binding
(``_capi.py``), a Python handle on a device-resident simulation
(``simulation.py``), the restart-file format (``state_io.py``) and seeded
initial conditions (``ics.py``).
"""
from . import ics  # noqa: F401  (pure numpy; importable without the library)

__all__ = ["ics", "Simulation", "make_params", "lib", "build_library"]


def build_library(verbose_ptxas: bool = False) -> str:
    from .build import build_library as _b
    return _b(verbose_ptxas)


def __getattr__(name):
    # the CUDA-backed names load the shared library on first use and raise
    # if it is missing (no CPU fallback exists)
    if name in ("Simulation", "make_params"):
        from . import simulation
        return getattr(simulation, name)
    if name == "lib":
        from ._capi import lib
        return lib
    raise AttributeError(name)
