"""One simulation sharded over several GPUs, one process per GPU.

Every rank holds a whole replica of the particle state (about 500 bytes per
particle: 0.5 GB at N = 1M).  The work that dominates a step is split:

* the leaf-parallel SPH loops -- the h solve with its neighbour lists, the
  density loop and the hydro loop -- run over a contiguous range of tree
  leaves per rank;
* direct-N gravity runs a contiguous share of the one-sided blocks and of the
  symmetric work items (tile pairs) per rank.

Three exchanges per step make every rank's state whole again, on the
context's stream, so all ranks continue with bit-identical state:

1. after the density loop: h, rho, div v, |curl v|, omega, psi and the
   neighbour count of every particle (64 bytes per particle).  Each
   particle's values come from the one rank whose leaves hold it, so an
   all-gather of the ranks' own slices makes the buffer whole (each byte
   crosses the links once; a sum would move it twice);
2. after the hydro loop: the accelerations and du/dt including the j-side
   pair forces a rank's pairs add to any particle (32 bytes), and the signal
   speeds (8 bytes);
3. after gravity: the gravitational accelerations and potentials (32 bytes).

Exchanges 2 and 3 are element-wise SUMs over the ranks (NCCL all-reduce) of
buffers in which a rank holds its own contributions and zeros elsewhere: a
rank's pairs reach particles of every rank, so these need the reduction.

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


def particle_spans(n: int, world: int) -> list[tuple[int, int]]:
    """The particles [lo, hi) whose SPH loops each rank runs (its leaves of 32)."""
    nleaf = (n + 31) // 32
    out = []
    for r in range(world):
        l0, l1 = shard_range(nleaf, r, world)
        out.append((min(l0 * 32, n), min(l1 * 32, n)))
    return out


def gather_owned(t, n: int, rank: int, world: int, group=None, work=None):
    """All-gather of the ranks' own particle slices of the flat per-particle
    buffer `t` (n x per values, this rank's slice valid): afterwards every
    rank holds every slice.  The slices are padded to the longest one for the
    collective and copied back in place.  `work`, if given, is a pair of
    reusable tensors (send, gathered) of the sizes this needs."""
    import torch
    import torch.distributed as dist
    per = t.numel() // max(n, 1)
    spans = particle_spans(n, world)
    chunk = max(hi - lo for lo, hi in spans) * per
    lo, hi = spans[rank]
    if work is None:
        work = (torch.empty(chunk, dtype=t.dtype, device=t.device),
                torch.empty(world * chunk, dtype=t.dtype, device=t.device))
    send, out = work
    send[(hi - lo) * per:chunk].zero_()
    send[:(hi - lo) * per].copy_(t[lo * per:hi * per])
    dist.all_gather_into_tensor(out, send, group=group)
    for r, (a, b) in enumerate(spans):
        if r != rank and b > a:
            t[a * per:b * per].copy_(out[r * chunk:r * chunk + (b - a) * per])
    return work


class ShardedSimulation(Simulation):
    """Shard `rank` of `world` of one simulation.

    ``reduce(tensor)`` sums a float64 CUDA tensor over the ranks in place,
    ordered on the torch stream that is current when it is called (the
    context's stream); the default is ``torch.distributed.all_reduce`` on the
    default process group (NCCL), and the density exchange is then an
    all-gather of the ranks' own slices (`gather_owned`).  A given ``reduce``
    takes all three exchanges (the zero-padded sums give the same result).
    Every rank must construct its shard from the same initial conditions and
    parameters and call ``step`` the same number of times."""

    def __init__(self, ic: dict, params, rank: int, world: int, device: int = 0, reduce=None):
        super().__init__(ic, params, device)
        check(lib().cudasph_set_shard(self._h, rank, world), "set_shard")
        self.rank, self.world = rank, world
        self._reduce = reduce
        self._stream = None
        self._gather_work = None

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
            elif name == "exchange":
                self._gather_work = gather_owned(t, self.n, self.rank, self.world, work=self._gather_work)
            else:
                import torch.distributed as dist
                dist.all_reduce(t)

    def step(self, k: int = 1):
        for _ in range(k):
            for names in self.stages():
                for name in names:
                    self._sum(name)
