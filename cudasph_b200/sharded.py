"""One simulation sharded over several GPUs, one process per GPU.

Every rank holds a whole replica of the particle state (about 500 bytes per
particle: 0.5 GB at N = 1M).  The work that dominates a step is split:

* the leaf-parallel SPH loops -- the h solve with its neighbour lists, the
  density loop and the hydro loop -- run over a contiguous range of tree
  leaves per rank;
* direct-N gravity runs a contiguous share of the one-sided blocks and of the
  symmetric work items (tile pairs) per rank.

Three exchanges per step make every rank's state whole again.  Each is an
element-wise SUM over the ranks of a buffer in which a rank holds its own
contributions and zeros elsewhere (an NCCL all-reduce on the context's
stream), so the sums are exact and all ranks continue with bit-identical
state:

1. after the density loop: h, rho, div v, |curl v|, omega, psi and the
   neighbour count of every particle (64 bytes per particle);
2. after the hydro loop: the accelerations and du/dt including the j-side
   pair forces a rank's pairs add to any particle (32 bytes), and the signal
   speeds (8 bytes);
3. after gravity: the gravitational accelerations and potentials (32 bytes).

The sort, predictor, tree, EOS, diagnostics, timestep and kick are cheap
per-particle or reduction passes and run replicated.  The reference runs one
GPU (its driver calls one device, CUDA_calls.cpp:3-26); this layer has no
counterpart there.
"""
from __future__ import annotations

import ctypes as C

from ._capi import check, lib
from .simulation import Simulation

BUFFERS = {"exchange": 0, "dots": 1, "vsig": 2, "grav": 3}


class _DeviceArray:
    """Zero-copy view of a device buffer (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def shard_range(count: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of [0, count) owned by shard `rank` of `world` (host code of the library)."""
    lo, hi = C.c_longlong(), C.c_longlong()
    check(lib().cudasph_shard_range(count, rank, world, C.byref(lo), C.byref(hi)), "shard_range")
    return lo.value, hi.value


class ShardedSimulation(Simulation):
    """Shard `rank` of `world` of one simulation.

    ``reduce(tensor)`` sums a float64 CUDA tensor over the ranks in place,
    ordered on the torch stream that is current when it is called (the
    context's stream); the default is ``torch.distributed.all_reduce`` on the
    default process group (NCCL).  Every rank must construct its shard from the
    same initial conditions and parameters and call ``step`` the same number
    of times."""

    def __init__(self, ic: dict, params, rank: int, world: int, device: int = 0, reduce=None):
        super().__init__(ic, params, device)
        check(lib().cudasph_set_shard(self._h, rank, world), "set_shard")
        self.rank, self.world = rank, world
        self._reduce = reduce
        self._stream = None

    def leaves(self) -> tuple[int, int]:
        """the leaf range [leaf0, leaf1) of this shard (after the first tree build)"""
        l0, l1 = C.c_int(), C.c_int()
        check(lib().cudasph_get_shard(self._h, None, None, C.byref(l0), C.byref(l1)), "get_shard")
        return l0.value, l1.value

    def buffer(self, name: str):
        """torch view of one exchanged buffer of the current state"""
        import torch
        ptr, cnt = C.c_void_p(), C.c_longlong()
        check(lib().cudasph_device_buffer(self._h, BUFFERS[name], C.byref(ptr), C.byref(cnt)), "device_buffer")
        return torch.as_tensor(_DeviceArray(ptr.value, cnt.value), device=f"cuda:{self.device}")

    def stages(self):
        """One step as a generator: runs the phases up to each exchange and
        yields the names of the buffers to sum over the ranks there."""
        L, h = lib(), self._h
        for name in ("begin_step", "predict", "build_tree", "solve_range", "density", "shard_pack"):
            check(getattr(L, "cudasph_" + name)(h), name)
        yield ("exchange",)
        for name in ("shard_unpack", "pressure", "hydro"):
            check(getattr(L, "cudasph_" + name)(h), name)
        yield ("dots", "vsig")
        check(L.cudasph_gravity(h), "gravity")
        yield ("grav",)
        for name in ("finish", "kick"):
            check(getattr(L, "cudasph_" + name)(h), name)

    def _sum(self, name: str):
        import torch
        t = self.buffer(name)
        with torch.cuda.stream(self.torch_stream()):
            if self._reduce is not None:
                self._reduce(t)
            else:
                import torch.distributed as dist
                dist.all_reduce(t)

    def step(self, k: int = 1):
        for _ in range(k):
            for names in self.stages():
                for name in names:
                    self._sum(name)
