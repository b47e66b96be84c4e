"""GPU parity of every phase of the step against the FP64 CPU oracle.

Integer work (Morton keys, the sort permutation, neighbour sets at a given
range) must match bit for bit.  The h solve, density and hydro loops are
compiled without FMA contraction and summed in the oracle's order (the oracle
is fed the particles in the GPU's tree order), so their FP64 results match to
a few ulp; the stated tolerances below leave room for library sqrt/cbrt/pow.
"""
import ctypes as C

import numpy as np
import pytest

from cudasph_b200 import ics
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sim(ic, **kw):
    from cudasph_b200.simulation import Simulation, make_params
    return Simulation(ic, make_params(**kw))


def _perm(ic, order):
    out = {}
    for k, v in ic.items():
        out[k] = np.asarray(v)[order] if isinstance(v, np.ndarray) and v.size == order.size else v
    return out


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def poly():
    ic = ics.polytrope(6000, n_ngb=50, seed=11)
    rs = np.random.default_rng(5)
    ic["vx"] = -0.3 * ic["y"] + rs.normal(0, 0.05, ic["x"].size)
    ic["vy"] = 0.3 * ic["x"] + rs.normal(0, 0.05, ic["x"].size)
    ic["vz"] = rs.normal(0, 0.05, ic["x"].size)
    return ic


def test_morton_keys_and_sort_bitexact():
    import torch
    from cudasph_b200._capi import check, lib
    rs = np.random.default_rng(1)
    n = 200_003
    x, y, z = (rs.normal(0, 1, n) for _ in range(3))
    x[:1000] = x[1000:2000]  # duplicate keys: ties must keep input order
    y[:1000] = y[1000:2000]
    z[:1000] = z[1000:2000]
    dev = torch.device("cuda:0")
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    box = torch.empty(4, dtype=torch.float64, device=dev)
    vals = torch.arange(n, dtype=torch.int32, device=dev)
    scratch = torch.empty(lib().cudasph_sort_scratch_bytes(n), dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    check(lib().cudasph_morton_keys(n, tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), keys.data_ptr(), box.data_ptr(), s))
    k_gpu = keys.cpu().numpy().view(np.uint64).copy()
    check(lib().cudasph_radix_sort_u64(n, keys.data_ptr(), vals.data_ptr(), scratch.data_ptr(), s))
    torch.cuda.synchronize()
    k_ref, box_ref = O.morton_keys(x, y, z)
    assert np.array_equal(k_gpu, k_ref)
    assert np.array_equal(box.cpu().numpy(), box_ref)
    order = O.sort_order(k_ref)
    assert np.array_equal(vals.cpu().numpy(), order)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), k_ref[order])


def test_peano_hilbert_keys_bitexact():
    """The reference's Peano-Hilbert curve on the GPU: the reference's own
    keys for 200 triplets (golden), the oracle's at every bit count 1..21
    (including coordinate bits above the key's range, which are ignored), and
    position keys with the reference's float quantisation."""
    import os
    import torch
    from cudasph_b200._capi import SphError, check, lib
    dev = torch.device("cuda:0")
    s = torch.cuda.current_stream().cuda_stream

    def gpu_keys(x, y, z, bits):
        t = [torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev) for a in (x, y, z)]
        k = torch.empty(len(x), dtype=torch.int64, device=dev)
        check(lib().cudasph_peano_hilbert_keys(len(x), t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), bits,
                                               k.data_ptr(), s))
        return k.cpu().numpy().view(np.uint64)

    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_tables.npz"))
    ph_in = gold["ph_in"]
    assert np.array_equal(gpu_keys(ph_in[:, 0], ph_in[:, 1], ph_in[:, 2], 18).view(np.int64), gold["ph_key"])
    rs = np.random.default_rng(9)
    for bits in range(1, 22):
        c = rs.integers(0, 1 << 31, size=(4000, 3))
        want = np.array([O.peano_hilbert_key(a, b, d, bits) for a, b, d in c], np.uint64)
        assert np.array_equal(gpu_keys(c[:, 0], c[:, 1], c[:, 2], bits), want), bits
    with pytest.raises(SphError):
        check(lib().cudasph_peano_hilbert_keys(1, 0, 0, 0, 22, 0, s))
    n = 200_003
    x, y, z = (rs.normal(0, 1, n) for _ in range(3))
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    box = torch.empty(4, dtype=torch.float64, device=dev)
    check(lib().cudasph_peano_keys(n, tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), keys.data_ptr(), box.data_ptr(), s))
    k_ref, box_ref = O.peano_keys(x, y, z)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), k_ref)
    assert np.array_equal(box.cpu().numpy(), box_ref)


def test_peano_key_mode_sorts_in_the_reference_order(poly):
    """key_mode = Peano-Hilbert: the context's sort is the stable order of
    the reference's keys, and a step in that order gives the same physics as
    one in Morton order (summation order only)."""
    sim = _sim(poly, n_target=50.0, eos_mode=0, soft_mode=1, eps=0.01, key_mode=1)
    sim.sort_bodies()
    k, _ = O.peano_keys(poly["x"], poly["y"], poly["z"])
    assert np.array_equal(sim.order(), O.sort_order(k))
    ref = _sim(poly, n_target=50.0, eos_mode=0, soft_mode=1, eps=0.01)
    sim.step(2)
    ref.step(2)
    assert np.array_equal(sim.n_ngb(), ref.n_ngb())
    for f in ("x", "vx", "rho", "ax", "du", "gx", "phi"):
        assert _rel(sim.get(f), ref.get(f)) < 1e-11, f
    sim.close()
    ref.close()


def test_sort_permutes_state(poly):
    sim = _sim(poly, n_target=50.0, eos_mode=0, soft_mode=1, eps=0.01)
    sim.sort_bodies()
    order = sim.order()
    k, _ = O.morton_keys(poly["x"], poly["y"], poly["z"])
    assert np.array_equal(order, O.sort_order(k))
    # fields come back in original order regardless of the tree order
    for f in ("x", "vx", "u", "m", "range"):
        assert np.array_equal(sim.get(f), poly[f])


def test_solve_range_matches_oracle(poly):
    sim = _sim(poly, n_target=50.0)
    sim.sort_bodies()
    order = sim.order()
    sim.CUDA_solve_range()
    r_gpu = sim.get("range")
    ev_gpu = sim.solve_evals()
    s = _perm(poly, order)
    r_orc, nn_orc, ev_orc = O.solve_range(s["x"], s["y"], s["z"], s["range"], O.make_params(n_target=50.0))
    r_orc_o = np.empty_like(r_orc)
    r_orc_o[order] = r_orc
    ev_o = np.empty_like(ev_orc)
    ev_o[order] = ev_orc
    exact = np.mean(r_gpu == r_orc_o)
    assert exact > 0.999, f"only {exact:.4f} of the ranges are bit-identical"
    assert np.max(np.abs(r_gpu / r_orc_o - 1)) < 2e-3
    assert np.mean(ev_gpu == ev_o) > 0.999


def test_find_ngb_sets_exact(poly):
    sim = _sim(poly, n_target=50.0)
    sim.CUDA_solve_range()
    sim.find_ngb()
    rng = sim.get("range")
    cnt, off, lst = sim.neighbours()
    c2, off2, lst2 = O.find_ngb(poly["x"], poly["y"], poly["z"], rng)
    assert np.array_equal(cnt, c2)
    for i in range(poly["x"].size):
        a = np.sort(lst[off[i]:off[i + 1]])
        b = lst2[off2[i]:off2[i + 1]]
        assert np.array_equal(a, b), f"particle {i}"
    assert sim.device_status() & 0x3 == 0


@pytest.mark.parametrize("eos", [0, 1])
def test_density_pressure_hydro_fp64(poly, eos):
    kw = dict(n_target=50.0, eos_mode=eos, soft_mode=0)
    sim = _sim(poly, **kw)
    sim.CUDA_solve_range()
    sim.find_ngb()
    sim.density()
    sim.pressure()
    sim.hydro()
    sim.synchronize()
    st = dict(poly)
    st["range"] = sim.get("range")
    cnt, off, lst = O.find_ngb(st["x"], st["y"], st["z"], st["range"])
    d = O.density(st, off, lst)
    for k in ("rho", "divv", "curlv", "omega", "psi"):
        assert _rel(sim.get(k), d[k]) < 1e-12, k
    st.update(d)
    p = O.make_params(**kw)
    st["P"] = O.pressure(st["rho"], st["u"], st["mu"], p)
    assert _rel(sim.get("P"), st["P"]) < 1e-12
    h = O.hydro(st, off, lst, p)
    for k in ("ax", "ay", "az", "du", "vsig"):
        assert _rel(sim.get(k), h[k]) < 1e-10, k


@pytest.mark.parametrize("soft", [0, 1])
def test_gravity_fp64(poly, soft):
    kw = dict(n_target=50.0, soft_mode=soft, eps=0.01)
    sim = _sim(poly, **kw)
    sim.CUDA_gravity()
    g = [sim.get(k) for k in ("gx", "gy", "gz", "phi")]
    ref = O.gravity(poly["x"], poly["y"], poly["z"], poly["m"], poly["range"], O.make_params(**kw))
    for a, b in zip(g, ref):
        assert _rel(a, b) < 1e-12


@pytest.mark.parametrize("soft", [0, 1])
def test_gravity_mixed_accuracy(poly, soft):
    kw = dict(n_target=50.0, soft_mode=soft, eps=0.01)
    sim = _sim(poly, precision=1, **kw)
    sim.CUDA_gravity()
    g = np.stack([sim.get(k) for k in ("gx", "gy", "gz")], 1)
    ref = O.gravity(poly["x"], poly["y"], poly["z"], poly["m"], poly["range"], O.make_params(**kw))
    r = np.stack(ref[:3], 1)
    rms = np.sqrt(np.mean(np.sum((g - r) ** 2, 1)) / np.mean(np.sum(r ** 2, 1)))
    assert rms < 1e-6
    assert _rel(sim.get("phi"), ref[3]) < 1e-5


@pytest.mark.parametrize("mask", [1, 2, 3])
def test_mixed_sph_pair_terms(poly, mask):
    """The FP32 density (bit 0) and hydro (bit 1) pair loops of the mixed
    form, against the FP64 step at the same state."""
    kw = dict(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)
    a = _sim(poly, precision=1, mixed_sph=mask, **kw)
    b = _sim(poly, **kw)
    a.step()
    b.step()
    assert np.max(np.abs(a.get("rho") / b.get("rho") - 1)) < (1e-6 if mask & 1 else 1e-12)
    ha = np.stack([a.get(k) - a.get(g) for k, g in (("ax", "gx"), ("ay", "gy"), ("az", "gz"))], 1)
    hb = np.stack([b.get(k) - b.get(g) for k, g in (("ax", "gx"), ("ay", "gy"), ("az", "gz"))], 1)
    rms = np.sqrt(np.mean(np.sum((ha - hb) ** 2, 1)) / np.mean(np.sum(hb ** 2, 1)))
    assert rms < 1e-5, rms
    assert _rel(a.get("du"), b.get("du")) < 1e-4
    assert a.device_status() & 0x7 == 0


def test_whole_steps_fp64_match_oracle():
    ic = ics.polytrope(3000, n_ngb=50, seed=3)
    kw = dict(n_target=50.0, eos_mode=0, soft_mode=1, eps=0.01)
    sim = _sim(ic, **kw)
    ref = O.Sim(ic, O.make_params(**kw))
    for _ in range(3):
        sim.step()
        ref.step()
    assert abs(sim.dt / ref.dt - 1) < 1e-9
    for k in ("x", "y", "z", "vx", "vy", "vz", "u", "range", "rho", "P", "ax", "du", "phi"):
        assert _rel(sim.get(k), ref.arr[k]) < 1e-8, k
    st = sim.system_statistics()
    so = ref.stats()
    assert abs(st["E"] - so[3]) < 1e-10 * abs(so[3])
    assert abs(st["time"] - ref.time) < 1e-15


@pytest.mark.parametrize("n", [40, 97, 1000, 2049])
def test_whole_steps_small_and_ragged_n_match_oracle(n):
    """Whole FP64 steps at sizes that reach the edges of the layout: a tree
    of one or two levels, a last leaf of fewer than 32 particles, a single
    gravity tile (the one-sided blocks then cover every pair) or one tile
    and a single particle beyond it, and a queue of resumed h-solve leaves
    that holds one leaf or none."""
    ic = ics.polytrope(n, n_ngb=24, seed=40 + n)
    kw = dict(n_target=24.0, eos_mode=1, soft_mode=1, eps=0.01)
    sim = _sim(ic, **kw)
    ref = O.Sim(ic, O.make_params(**kw))
    for _ in range(3):
        sim.step()
        ref.step()
    for k in ("x", "vx", "u", "range", "rho", "P", "ax", "du", "phi"):
        assert _rel(sim.get(k), ref.arr[k]) < 1e-8, (n, k)
    assert np.array_equal(sim.n_ngb(), ref.n_ngb)
    assert sim.device_status() & 0x7 == 0
    sim.close()


def test_graph_replay_matches_eager_steps():
    ic = ics.polytrope(5000, n_ngb=50, seed=9)
    kw = dict(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01, precision=1)
    a = _sim(ic, **kw)
    b = _sim(ic, **kw)
    b.set_graph(True)
    for _ in range(5):  # step 1 sorts from the IC (eager); 2, 3 capture; 4, 5 replay
        a.step()
        b.step()
    for k in ("x", "vx", "u", "range", "rho", "ax", "phi"):
        assert _rel(b.get(k), a.get(k)) < 1e-11, k
    assert abs(b.time - a.time) <= 1e-14 * abs(a.time)
    assert b.kernel_launches() == a.kernel_launches()


def test_step_through_host_buffers_matches_the_resident_step(poly):
    """cudasph_step_host (state in from host buffers, one step, state out, the
    end-to-end path of the bench) and the batched set/get_state entries give
    the same step as the device-resident handle."""
    from cudasph_b200._capi import FIELDS
    kw = dict(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)
    a = _sim(poly, **kw)
    a.step()
    ins = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu")
    b = _sim(poly, **kw)
    src = {k: np.ascontiguousarray(poly[k], np.float64) for k in ins}
    out = {k: np.full(poly["x"].size, np.nan) for k in FIELDS}
    b.step_host(src, out)
    for k in ("x", "vx", "u", "range", "rho", "P", "ax", "du", "gx", "phi", "vsig"):
        assert _rel(out[k], a.get(k)) < 1e-12, k
    got = {k: np.empty(poly["x"].size) for k in ("x", "rho", "ax")}
    b.get_state_host(got)
    for k in got:
        assert np.array_equal(got[k], out[k]), k
    b.set_state_host({"u": 2 * out["u"]})
    assert np.array_equal(b.get("u"), 2 * out["u"])
    a.close()
    b.close()
