"""The sharded step (cudasph_set_shard, cudasph_b200.sharded) on one GPU.

W shards of one simulation -- W contexts, each on its own stream -- are
stepped phase by phase in lockstep, and the three exchanges are done as
element-wise sums of the shards' device buffers, which is what the NCCL
all-reduce does across GPUs.  Kernels of different shards never wait on one
another: each exchange synchronizes every shard's stream first.  The result
must equal the unsharded step (neighbour counts exactly; FP64 fields to the
rounding of FP64 atomics added in another order), and all shards must hold
bit-identical state; FP64, mixed, unequal masses, spline softening and the
tree gravity are covered.  A one-rank NCCL process group runs the same
protocol through torch.distributed on the context's stream.
"""
import numpy as np
import pytest

from cudasph_b200 import ics

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "range", "vx", "vy", "vz", "u", "rho", "P", "divv", "curlv", "omega", "psi", "ax", "ay",
          "az", "du", "gx", "gy", "gz", "phi", "vsig")


def _ic(n=20000, seed=31, equal=True):
    ic = ics.polytrope(n, n_ngb=50, seed=seed)
    rs = np.random.default_rng(seed)
    ic["vx"] = -0.3 * ic["y"] + rs.normal(0, 0.05, n)
    ic["vy"] = 0.3 * ic["x"] + rs.normal(0, 0.05, n)
    ic["vz"] = rs.normal(0, 0.05, n)
    if not equal:
        ic["m"] = ic["m"] * rs.uniform(0.5, 1.5, n)
    return ic


def _lockstep(shards, steps):
    import torch
    for _ in range(steps):
        gens = [s.stages() for s in shards]
        while True:
            names = [next(g, None) for g in gens]
            if names[0] is None:
                assert all(x is None for x in names)
                break
            assert all(x == names[0] for x in names)
            for s in shards:
                s.synchronize()
            for name in names[0]:
                bufs = [s.buffer(name) for s in shards]
                tot = bufs[0].clone()
                for b in bufs[1:]:
                    tot += b
                for b in bufs:
                    b.copy_(tot)
            torch.cuda.synchronize()


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("precision,soft,equal,grav", [(0, 1, True, 0), (1, 1, True, 0), (1, 1, False, 0),
                                                       (1, 0, True, 0), (1, 1, True, 1)])
def test_lockstep_shards_equal_unsharded_step(world, precision, soft, equal, grav):
    from cudasph_b200.sharded import ShardedSimulation
    from cudasph_b200.simulation import Simulation, make_params
    ic = _ic(equal=equal)
    par = dict(precision=precision, n_target=50.0, eos_mode=1, soft_mode=soft, eps=0.01, grav_mode=grav)
    ref = Simulation(ic, make_params(**par))
    shards = [ShardedSimulation(ic, make_params(**par), r, world) for r in range(world)]
    ref.step()
    _lockstep(shards, 1)
    nref = ref.n_ngb()
    spans = [s.leaves() for s in shards]
    assert spans[0][0] == 0 and all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    for s in shards:
        assert np.array_equal(s.n_ngb(), nref)
    ref.step()
    _lockstep(shards, 1)
    got = [{k: s.get(k) for k in FIELDS} for s in shards]
    for g in got[1:]:
        for k in FIELDS:
            assert np.array_equal(g[k], got[0][k]), k
    for k in FIELDS:
        assert _rel(got[0][k], ref.get(k)) < 1e-9, k
    assert abs(shards[0].dt - ref.dt) <= 1e-12 * ref.dt
    for s in shards:
        assert s.device_status() == 0
        s.close()
    ref.close()


def test_sharded_context_refuses_whole_step_and_adjoint():
    from cudasph_b200._capi import SphError
    from cudasph_b200.sharded import ShardedSimulation
    from cudasph_b200.simulation import make_params
    s = ShardedSimulation(_ic(n=3000), make_params(n_target=50.0, soft_mode=1, eps=0.01), 1, 2)
    with pytest.raises(SphError):
        s._call("step")
    with pytest.raises(SphError):
        s.set_keep(True)
    s.close()


def test_one_rank_nccl_group_runs_the_sharded_step():
    import os
    import socket
    import torch.distributed as dist
    from cudasph_b200.sharded import ShardedSimulation
    from cudasph_b200.simulation import Simulation, make_params
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        ic = _ic(n=20000)
        par = dict(precision=1, n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)
        ref = Simulation(ic, make_params(**par))
        sh = ShardedSimulation(ic, make_params(**par), 0, 1)
        ref.step(2)
        sh.step(2)
        sh.synchronize()
        for k in FIELDS:
            assert _rel(sh.get(k), ref.get(k)) < 1e-9, k
        sh.close()
        ref.close()
    finally:
        dist.destroy_process_group()
