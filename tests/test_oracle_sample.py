"""The oracle's sampled-target loops (used to check the GPU at full workload
sizes) against its whole-set loops on a small state: the h solve, the
neighbour sets and the density loop bit for bit, the hydro derivatives (i-side
plus the j-side scatter) to the rounding of a different summation order."""
import numpy as np

from cudasph_b200 import ics
from oracle import oracle as O


def test_sampled_loops_equal_the_whole_set_loops():
    n = 4000
    ic = ics.polytrope(n, n_ngb=50, seed=3)
    rs = np.random.default_rng(1)
    for k in ("vx", "vy", "vz"):
        ic[k] = rs.normal(0, 0.1, n)
    p = O.make_params(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)
    r, nn, ne = O.solve_range(ic["x"], ic["y"], ic["z"], ic["range"], p)
    tg = np.sort(rs.choice(n, 300, replace=False))
    r2, nn2, ne2 = O.solve_range_sample(ic["x"], ic["y"], ic["z"], ic["range"], tg, p)
    assert np.array_equal(r[tg], r2) and np.array_equal(nn[tg], nn2) and np.array_equal(ne[tg], ne2)
    cnt, off, lst = O.find_ngb(ic["x"], ic["y"], ic["z"], r)
    c2, o2, l2 = O.find_ngb_sample(ic["x"], ic["y"], ic["z"], r[tg], tg)
    assert np.array_equal(cnt[tg], c2)
    for t, i in enumerate(tg):
        assert np.array_equal(lst[off[i]:off[i + 1]], l2[o2[t]:o2[t + 1]])
    st = dict(ic, range=r)
    d = O.density(st, off, lst)
    d2 = O.density_sample(st, tg, o2, l2)
    for k in d:
        assert np.array_equal(d[k][tg], d2[k]), k
    st.update(d)
    st["P"] = O.pressure(st["rho"], st["u"], st["mu"], p)
    h = O.hydro(st, off, lst, p)
    h2 = O.hydro_sample(st, tg, p)
    for k in ("ax", "ay", "az"):
        assert np.max(np.abs(h[k][tg] - h2[k])) <= 1e-13 * np.max(np.abs(h[k][tg])), k
    for k in ("du", "vsig"):
        assert np.array_equal(h[k][tg], h2[k]), k


def test_sampled_parity_of_the_oracle_with_itself():
    """oracle/checks.sampled_parity fed the oracle's own whole-set results
    reports zero error (and sees a planted error in one density value)."""
    from oracle import checks
    n = 3000
    ic = ics.polytrope(n, n_ngb=50, seed=5)
    p = O.make_params(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)
    st_in = {k: np.asarray(ic[k], np.float64) for k in checks.STATE_IN}
    r, nn, _ = O.solve_range(ic["x"], ic["y"], ic["z"], ic["range"], p)
    cnt, off, lst = O.find_ngb(ic["x"], ic["y"], ic["z"], r)
    st = dict(ic, range=r)
    st.update(O.density(st, off, lst))
    st["P"] = O.pressure(st["rho"], st["u"], st["mu"], p)
    st.update(O.hydro(st, off, lst, p))
    g = O.gravity(ic["x"], ic["y"], ic["z"], ic["m"], r, p)
    for k, a in zip(("gx", "gy", "gz", "phi"), g):
        st[k] = a
    st_out = {k: np.asarray(st[k], np.float64) for k in checks.STATE_OUT}
    tg = np.arange(0, n, 7, dtype=np.int32)
    lists = [lst[off[i]:off[i + 1]] for i in tg]
    res = checks.sampled_parity(st_in, st_out, tg, p, n_ngb=cnt, lists=lists, grav_targets=tg[::2])
    assert res["h_identical_frac"] == 1.0 and res["list_mismatch"] == 0 and res["n_ngb_mismatch"] == 0
    for k in ("rho", "divv", "curlv", "omega", "psi", "P", "du", "vsig", "gravity", "phi"):
        assert res[f"{k}_max_rel"] == 0.0, k
    assert res["hydro_rms_rel"] < 1e-14
    st_out["rho"] = st_out["rho"].copy()
    st_out["rho"][tg[3]] *= 1 + 1e-9
    assert checks.sampled_parity(st_in, st_out, tg, p, grav_targets=tg[:4])["rho_max_rel"] > 1e-10
