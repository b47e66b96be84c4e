"""The oracle as the checker of one force evaluation of the GPU step at full
workload size, on a seeded sample of target particles.

TEST INFRASTRUCTURE: used by tests/ and by the cpu_baseline leg of bench.py.
The product (cudasph_b200) never imports it.

A force evaluation is the middle of one step (step.cpp:62-103): the h solve
(dev_solve_range.cu:174-189), the neighbour sets (dev_find_ngb.cu:13-87), the
density loop (dev_density_loop.cu:29-111), the EOS (dev_compute_pressure.cu:
99-111), the hydro derivatives with viscosity and the j-side scatter
(dev_hydro_dots.cu:25-113, sph_accelerations.cpp:106-114) and the gravity
(sph_grav_kernel.cu:14-111).  Every array handed in is in the GPU's tree order
(slot order), so that the oracle's candidates and lists, ascending in index,
come in the same order as the GPU's and the FP64 sums can agree to the last
bit.  The per-particle inputs of the hydro and gravity checks (range, rho, P,
div v, curl v, omega, psi of every particle) are the GPU's own: each loop is
checked on the state the GPU gave it, and the per-particle fields are checked
on the sample.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

STATE_IN = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu")
STATE_OUT = ("range", "rho", "divv", "curlv", "omega", "psi", "P", "ax", "ay", "az", "du", "vsig", "gx", "gy",
             "gz", "phi")


def slot_lists(order, cnt, off, lst, slots):
    """GPU neighbour lists (original ids, CSR over original ids) of the given
    tree slots, as ascending slot indices."""
    inv = np.empty(order.size, np.int64)
    inv[order] = np.arange(order.size)
    out = []
    for s in slots:
        o = order[s]
        out.append(np.sort(inv[lst[off[o]:off[o + 1]]]))
    return out


def _maxrel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _rms3(a, b):
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, 1)) / np.mean(np.sum(b ** 2, 1))))


def sampled_parity(st_in: dict, st_out: dict, targets, params: "O.OrcParams", n_ngb=None, lists=None,
                   grav_targets=None, hydro_total: bool = False) -> dict:
    """Errors of one GPU force evaluation against the oracle on `targets`
    (tree slots).

    st_in: the state the evaluation started from (positions, velocities and u
      after the predictor, masses, mu, and `range` = the h solve's starting
      guess); st_out: the GPU's results (range after the solve, density
      fields, P, ax..du (hydro only, or hydro + gravity if hydro_total), vsig,
      gravity).  n_ngb: the GPU's hard counts (slot order); lists: the GPU's
      lists of the targets (slot_lists).  grav_targets: the targets of the
      gravity check (default: the first 2048 of `targets`)."""
    t = np.ascontiguousarray(targets, np.int32)
    res = {"targets": int(t.size)}
    # h solve from the same guess, against all particles
    r_o, nn_o, _ = O.solve_range_sample(st_in["x"], st_in["y"], st_in["z"], st_in["range"], t, params)
    r_g = st_out["range"][t]
    same = r_g == r_o
    res["h_identical_frac"] = float(np.mean(same))
    res["h_max_rel"] = float(np.max(np.abs(r_g / r_o - 1)))
    # neighbour sets at the GPU's ranges: exact
    cnt_o, off_o, lst_o = O.find_ngb_sample(st_in["x"], st_in["y"], st_in["z"], r_g, t)
    if n_ngb is not None:
        res["n_ngb_mismatch"] = int(np.sum(n_ngb[t] != cnt_o))
        # the solve's own count at its final range, where the two ranges agree
        res["n_ngb_solve_mismatch"] = int(np.sum((n_ngb[t] != nn_o) & same))
    if lists is not None:
        res["list_mismatch"] = int(sum(not np.array_equal(lists[k], lst_o[off_o[k]:off_o[k + 1]])
                                       for k in range(t.size)))
    # density at the GPU's ranges over the oracle's lists
    s = dict(st_in)
    s["range"] = st_out["range"]
    d = O.density_sample(s, t, off_o, lst_o)
    for k in ("rho", "divv", "curlv", "omega", "psi"):
        res[f"{k}_max_rel"] = _maxrel(st_out[k][t], d[k])
    # EOS on the GPU's density
    P = O.pressure(st_out["rho"][t], st_in["u"][t], st_in["mu"][t], params)
    res["P_max_rel"] = _maxrel(st_out["P"][t], P)
    # hydro over the GPU's per-particle fields
    for k in ("rho", "divv", "curlv", "omega", "psi", "P"):
        s[k] = st_out[k]
    h = O.hydro_sample(s, t, params)
    grav_targets = t[:2048] if grav_targets is None else np.ascontiguousarray(grav_targets, np.int32)
    g = O.gravity(st_in["x"], st_in["y"], st_in["z"], st_in["m"], st_out["range"], params, targets=grav_targets)
    g_gpu = np.stack([st_out[k][grav_targets] for k in ("gx", "gy", "gz")], 1)
    g_orc = np.stack(g[:3], 1)
    res["gravity_targets"] = int(grav_targets.size)
    res["gravity_rms_rel"] = _rms3(g_gpu, g_orc)
    res["gravity_max_rel"] = _maxrel(g_gpu, g_orc)
    res["phi_max_rel"] = _maxrel(st_out["phi"][grav_targets], g[3])
    a_gpu = np.stack([st_out[k][t] for k in ("ax", "ay", "az")], 1)
    a_orc = np.stack([h[k] for k in ("ax", "ay", "az")], 1)
    if hydro_total:
        # ax..az hold hydro + gravity: the hydro part is checked on the
        # gravity targets, where the oracle has both
        pos = {int(v): k for k, v in enumerate(t)}
        sel = np.array([pos[int(v)] for v in grav_targets])
        tot_o = a_orc[sel] + g_orc
        res["force_rms_rel"] = _rms3(a_gpu[sel], tot_o)
        res["hydro_rms_rel"] = _rms3(a_gpu[sel] - g_gpu, a_orc[sel])
    else:
        for c, k in enumerate(("ax", "ay", "az")):
            res[f"{k}_max_rel"] = _maxrel(a_gpu[:, c], a_orc[:, c])
        res["hydro_rms_rel"] = _rms3(a_gpu, a_orc)
        sel = np.searchsorted(t, grav_targets) if np.all(np.diff(t) > 0) else None
        if sel is not None and np.array_equal(t[sel], grav_targets):
            res["force_rms_rel"] = _rms3(a_gpu[sel] + g_gpu, a_orc[sel] + g_orc)
    res["du_max_rel"] = _maxrel(st_out["du"][t], h["du"])
    res["vsig_max_rel"] = _maxrel(st_out["vsig"][t], h["vsig"])
    return res


def capture_force_evaluation(sim):
    """Run one force evaluation of the step on a Simulation phase by phase
    (begin_step's sort, predict, sph_accelerations, gravity; no finish or
    kick) and return (st_in, st_out, n_ngb, order) in tree order."""
    from cudasph_b200._capi import check, lib
    check(lib().cudasph_begin_step(sim._h), "begin_step")
    sim.predict()
    order = sim.order()
    st_in = {k: sim.get(k)[order] for k in STATE_IN}
    sim.sph_accelerations()
    sim.CUDA_gravity()
    sim.synchronize()
    st_out = {k: sim.get(k)[order] for k in STATE_OUT}
    return st_in, st_out, sim.n_ngb()[order], order
