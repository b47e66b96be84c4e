"""The sharded step's decomposition and exchanges on two CPU ranks (gloo).

A sharded context (cudasph_set_shard) runs the leaf-parallel SPH loops over
its contiguous leaf range and its share of the gravity blocks, and three
element-wise sums over the ranks make the state whole (cudasph_b200.sharded).
Here two gloo ranks play that protocol with the FP64 oracle as the compute
engine, over the library's own partition (cudasph_shard_range):

1. each rank packs the h-solve and density results of its own particles
   (zeros elsewhere); the sum is every particle's values, bit for bit;
2. each rank runs the hydro loop over its own particles' lists only -- the
   i-side sums and the j-side pair forces those pairs add to any particle
   (sph_accelerations.cpp:106-114) -- and the sum equals the whole hydro
   pass up to the order of the FP64 additions;
3. each rank computes gravity for its own block of targets; the sum equals
   the whole gravity pass bit for bit;
and both ranks end with identical buffers.  No GPU is used.
"""
import os
import socket

import numpy as np
import pytest

from cudasph_b200 import ics
from oracle import oracle as O

WORLD = 2
KLEAF = 32


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _csr_own(off, lst, lo, hi):
    """The lists of particles [lo, hi) only (other particles get empty lists)."""
    n = off.size - 1
    cnt = np.diff(off)
    keep = np.zeros(n, bool)
    keep[lo:hi] = True
    cnt2 = np.where(keep, cnt, 0)
    off2 = np.zeros(n + 1, np.int64)
    off2[1:] = np.cumsum(cnt2)
    lst2 = lst[off[lo]:off[hi]].copy()
    return off2, lst2


def _rank_main(rank, port, out_dir):
    import torch
    import torch.distributed as dist
    from cudasph_b200.sharded import shard_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        ic = ics.polytrope(3000, n_ngb=50, seed=17)
        rs = np.random.default_rng(3)
        for k in ("vx", "vy", "vz"):
            ic[k] = rs.normal(0, 0.1, ic["x"].size)
        n = ic["x"].size
        par = O.make_params(n_target=50.0, eos_mode=1, soft_mode=0)
        # replicated (deterministic): h solve and lists of every particle
        rng, _, _ = O.solve_range(ic["x"], ic["y"], ic["z"], ic["range"], par)
        cnt, off, lst = O.find_ngb(ic["x"], ic["y"], ic["z"], rng)
        s = dict(ic, range=rng)
        nleaf = (n + KLEAF - 1) // KLEAF
        l0, l1 = shard_range(nleaf, rank, WORLD)
        lo, hi = l0 * KLEAF, min(l1 * KLEAF, n)

        # 1. SPH exchange: own h-solve + density results, zeros elsewhere
        d = O.density(s, off, lst)
        cols = [rng, d["rho"], d["divv"], d["curlv"], d["omega"], d["psi"], cnt.astype(np.float64)]
        full = np.stack(cols, 1)
        x = np.zeros_like(full)
        x[lo:hi] = full[lo:hi]
        t = torch.from_numpy(x)
        dist.all_reduce(t)
        xsum = t.numpy()
        s.update(rho=xsum[:, 1], divv=xsum[:, 2], curlv=xsum[:, 3], omega=xsum[:, 4], psi=xsum[:, 5])
        s["P"] = O.pressure(s["rho"], s["u"], s["mu"], par)

        # 2. hydro over own lists (i-side + j-side of own pairs)
        off_o, lst_o = _csr_own(off, lst, lo, hi)
        h = O.hydro(s, off_o, lst_o, par)
        hs = {}
        for k in ("ax", "ay", "az", "du", "vsig"):
            t = torch.from_numpy(h[k].copy())
            dist.all_reduce(t)
            hs[k] = t.numpy()
        href = O.hydro(s, off, lst, par)

        # 3. gravity: own block of targets (the one-sided decomposition)
        nb = (n + 255) // 256
        b0, b1 = shard_range(nb, rank, WORLD)
        tg = np.arange(b0 * 256, min(b1 * 256, n), dtype=np.int32)
        g = O.gravity(ic["x"], ic["y"], ic["z"], ic["m"], rng, par, targets=tg)
        gbuf = np.zeros((n, 4))
        gbuf[tg] = np.stack(g, 1)
        t = torch.from_numpy(gbuf)
        dist.all_reduce(t)
        gsum = t.numpy()
        gref = np.stack(O.gravity(ic["x"], ic["y"], ic["z"], ic["m"], rng, par), 1)

        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), xsum=xsum, full=full, gsum=gsum, gref=gref,
                 own=np.array([lo, hi]), **{"h_" + k: v for k, v in hs.items()},
                 **{"r_" + k: href[k] for k in hs})
    finally:
        dist.destroy_process_group()


def test_sharded_exchanges_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(port, str(tmp_path)), nprocs=WORLD, join=True, start_method="spawn")
    r = [np.load(tmp_path / f"rank{k}.npz") for k in range(WORLD)]
    # the two ranks own complementary, non-empty leaf ranges
    assert r[0]["own"][0] == 0 and r[0]["own"][1] == r[1]["own"][0] and r[1]["own"][1] == r[0]["full"].shape[0]
    assert r[0]["own"][1] > 0 and r[1]["own"][1] > r[1]["own"][0]
    for k in r[0].files:  # identical state on both ranks
        if k != "own":
            assert np.array_equal(r[0][k], r[1][k]), k
    a = r[0]
    assert np.array_equal(a["xsum"], a["full"])
    assert np.array_equal(a["gsum"], a["gref"])
    for k in ("ax", "ay", "az", "du"):
        ref = a["r_" + k]
        assert np.max(np.abs(a["h_" + k] - ref)) <= 1e-12 * np.max(np.abs(ref)), k
    assert np.array_equal(a["h_vsig"], a["r_vsig"])


@pytest.mark.parametrize("count", [0, 1, 5, 31, 1000, 65921])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_range_partitions(count, world):
    from cudasph_b200.sharded import shard_range
    spans = [shard_range(count, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == count
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0
    sizes = [h - l for l, h in spans]
    assert min(sizes) >= 0 and max(sizes) - min(sizes) <= 1
