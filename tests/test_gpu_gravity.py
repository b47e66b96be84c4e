"""Direct-N gravity through the standalone entry point cudasph_gravity_direct.

The mixed Plummer form computes each pair once above the diagonal tiles of
1,024 particles (work items of up to 8, 4, 2 or 1 tiles: the most that still
gives four items per SM) and the diagonal tiles one-sided, so the sizes below
cover: a single tile, an exact tile, a ragged second tile, rows split over
several work items with a ragged last batch, and each item length.
Reference: the FP64 oracle restatement of sph_grav_kernel.cu:14-111 (Plummer
mode) on the same particles.
"""
import numpy as np
import pytest

from oracle import known_answers as KA
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [1000, 1024, 1025, 2048, 5000, 20001]


def _cloud(n, seed, condensed=False):
    rs = np.random.default_rng(seed)
    # a uniform ball, or a centrally condensed cloud; both with coincident pairs
    r = rs.random(n) ** 2 if condensed else rs.random(n) ** (1.0 / 3.0)
    v = rs.normal(size=(n, 3))
    p = v / np.linalg.norm(v, axis=1)[:, None] * r[:, None]
    p[1::97] = p[0::97][: p[1::97].shape[0]]
    m = rs.uniform(0.5, 1.5, n) / n
    return p, m


def _run(p, m, eps, G, precision):
    import torch
    from cudasph_b200._capi import lib
    n = m.size
    src = torch.from_numpy(np.column_stack([p, m]).astype(np.float64).copy()).cuda()
    out = torch.full((n, 4), np.nan, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib().cudasph_gravity_direct(n, src.data_ptr(), None, out.data_ptr(), 1, eps, G, precision, st)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle(p, m, eps, G):
    par = O.make_params(soft_mode=1, eps=eps, G=G)
    g = O.gravity(p[:, 0], p[:, 1], p[:, 2], m, np.zeros_like(m), par)
    return np.stack(g, 1)


# RMS force error bound of the mixed form, 1e-5: FP32 pair terms give 1e-6 to
# 6e-6 on these clouds (their net forces cancel strongly, and close pairs lose
# digits to FP32 rounding of the anchor-relative coordinates) on both the
# one-sided (n <= 1024) and the symmetric path; a pair missed or counted twice
# shows as 1e-3 or more.
@pytest.mark.parametrize("condensed,bound", [(False, 1e-5), (True, 1e-5)])
@pytest.mark.parametrize("n", SIZES)
def test_mixed_plummer_gravity_matches_oracle(n, condensed, bound):
    p, m = _cloud(n, 100 + n, condensed)
    eps, G = 0.004, 1.3
    got = _run(p, m, eps, G, 1)
    ref = _oracle(p, m, eps, G)
    assert np.all(np.isfinite(got))
    a, r = got[:, :3], ref[:, :3]
    rms = np.sqrt(np.mean(np.sum((a - r) ** 2, 1)) / np.mean(np.sum(r ** 2, 1)))
    assert rms < bound, rms
    assert np.max(np.abs(got[:, 3] / ref[:, 3] - 1)) < 1e-5


@pytest.mark.parametrize("n", [1025, 20001])
def test_fp64_plummer_gravity_matches_oracle(n):
    p, m = _cloud(n, 7 + n)
    got = _run(p, m, 0.004, 1.0, 0)
    ref = _oracle(p, m, 0.004, 1.0)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


# Item lengths by N: 20,001 (20 tiles) takes single-tile items, 65,536 (64)
# two, 71,380 (70, ragged) four, 97,000 (95, ragged) eight.  Checked on 512
# sampled targets against the oracle's sum over all sources.
@pytest.mark.parametrize("n", [65536, 71380, 97000])
@pytest.mark.parametrize("precision", [0, 1])
def test_gravity_item_lengths_match_oracle(n, precision):
    p, m = _cloud(n, 11 + n)
    got = _run(p, m, 0.004, 1.0, precision)
    tg = np.sort(np.random.default_rng(n).choice(n, 512, replace=False)).astype(np.int32)
    par = O.make_params(soft_mode=1, eps=0.004, G=1.0)
    ref = np.stack(O.gravity(p[:, 0], p[:, 1], p[:, 2], m, np.zeros_like(m), par, targets=tg), 1)
    g = got[tg]
    assert np.all(np.isfinite(got))
    if precision == 0:
        assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))
    else:
        a, r = g[:, :3], ref[:, :3]
        assert np.sqrt(np.mean(np.sum((a - r) ** 2, 1)) / np.mean(np.sum(r ** 2, 1))) < 1e-5
        assert np.max(np.abs(g[:, 3] / ref[:, 3] - 1)) < 1e-5


def test_mixed_pair_forces_conserve_momentum():
    # each off-diagonal pair applies equal and opposite FP32 forces
    p, m = _cloud(20001, 3)
    got = _run(p, m, 0.004, 1.0, 1)
    ma = got[:, :3] * m[:, None]
    assert np.linalg.norm(ma.sum(0)) < 1e-6 * np.abs(ma).sum()


# The step's gravity phase takes the equal-mass form of the symmetric kernels
# (the mass factored out of both pair sums) when every mass equals the first,
# a flag computed on the device with the gravity sources; otherwise the
# general form.  Both must agree with the standalone entry point, which always
# runs the general form, and with the oracle.  n = 5000 gives five 1,024-tiles
# (symmetric items plus a ragged last tile whose padding sources the
# equal-mass form parks far away).
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("equal", [True, False])
def test_step_gravity_equal_mass_form(precision, equal):
    from cudasph_b200 import ics
    from cudasph_b200.simulation import Simulation, make_params
    ic = ics.polytrope(5000, n_ngb=50, seed=21)
    if not equal:
        ic["m"] = ic["m"] * np.random.default_rng(2).uniform(0.5, 1.5, ic["m"].size)
    eps, G = 0.004, 1.3
    sim = Simulation(ic, make_params(precision=precision, n_target=50.0, soft_mode=1, eps=eps, G=G))
    sim.CUDA_gravity()
    got = np.stack([sim.get(k) for k in ("gx", "gy", "gz", "phi")], 1)
    order = sim.order()  # the step computes in its own (input or tree) order
    sim.close()
    p = np.stack([ic["x"], ic["y"], ic["z"]], 1)
    gen = np.empty_like(got)
    gen[order] = _run(p[order], ic["m"][order], eps, G, precision)
    ref = _oracle(p, ic["m"], eps, G)
    assert np.all(np.isfinite(got))
    a, g, r = got[:, :3], gen[:, :3], ref[:, :3]
    if precision == 0:
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
        assert np.max(np.abs(got - gen)) <= 1e-13 * np.max(np.abs(ref))
    else:
        rms = lambda x, y: np.sqrt(np.mean(np.sum((x - y) ** 2, 1)) / np.mean(np.sum(y ** 2, 1)))
        assert rms(a, r) < 1e-6
        assert rms(a, g) < 1e-6
        # the equal-mass form's padding sources carry no potential weight:
        # their 1/s of about 1e-18 must not show in any particle's potential
        assert np.max(np.abs(got[:, 3] / ref[:, 3] - 1)) < 1e-6


# Isolated pairs through the standalone gravity entry against the closed-form
# softened law (oracle/known_answers.py): Plummer and the spline softening at
# the ranges 0.2 and 0.3, in every regime of r (inner and outer polynomial of
# each range, between them, beyond both) and for coincident particles.  FP64
# to the 12-decimal constants of the spline polynomials; mixed to FP32.
PAIR_SEPARATIONS = [0.0, 0.01, 0.05, 0.099, 0.101, 0.149, 0.151, 0.199, 0.201, 0.25, 0.299, 0.301, 0.6]


@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 1e-5)])
@pytest.mark.parametrize("soft_mode", [0, 1])
def test_isolated_pair_follows_the_softening_law(soft_mode, precision, tol):
    import torch
    from cudasph_b200._capi import lib
    eps, G = 0.05, 1.3
    st = torch.cuda.current_stream().cuda_stream
    for r in PAIR_SEPARATIONS:
        pos, m, rng, acc, phi = KA.two_body(r, soft_mode=soft_mode, eps=eps, G=G)
        src = torch.from_numpy(np.column_stack([pos, m]).copy()).cuda()
        ranges = torch.from_numpy(rng.copy()).cuda()  # the entry squares them on the device
        out = torch.full((2, 4), np.nan, dtype=torch.float64, device="cuda")
        rc = lib().cudasph_gravity_direct(2, src.data_ptr(), ranges.data_ptr() if soft_mode == 0 else None,
                                          out.data_ptr(), soft_mode, eps, G, precision, st)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), r
        if r == 0.0:
            assert np.all(got[:, :3] == 0.0)
        else:
            assert np.max(np.abs(got[:, :3] - acc)) <= tol * np.max(np.abs(acc)), (r, got[:, :3], acc)
        assert np.max(np.abs(got[:, 3] / phi - 1)) <= tol, (r, got[:, 3], phi)
