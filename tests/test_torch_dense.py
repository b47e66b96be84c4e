"""The dense FP64 PyTorch restatement (the adjoint's reference) against the C
oracle (forward) and against central finite differences (gradients).  CPU."""
import numpy as np
import pytest
import torch

from cudasph_b200 import ics
from oracle import oracle as O
from oracle import torch_dense as T


def _ic(n, seed):
    ic = ics.polytrope(n, n_ngb=32, seed=seed)
    rs = np.random.default_rng(seed)
    ic["vx"] = -0.2 * ic["y"] + rs.normal(0, 0.03, n)
    ic["vy"] = 0.2 * ic["x"] + rs.normal(0, 0.03, n)
    ic["vz"] = rs.normal(0, 0.03, n)
    return ic


def test_dense_forward_matches_oracle():
    ic = _ic(400, 4)
    sim = O.Sim(ic, O.make_params(n_target=32.0, eos_mode=1, soft_mode=1, eps=0.01, rel_err=1e-13, max_iter=80))
    sim.step()
    sim.step()
    st = T.state_from_ic(ic)
    p = T.default_params(n_target=32.0, eos_mode=1, eps=0.01)
    for _ in range(2):
        st = T.step(st, p)
    for k, ref in (("x", sim.arr["x"]), ("w", sim.arr["range"]), ("rho", sim.arr["rho"]), ("P", sim.arr["P"]),
                   ("du", sim.arr["du"])):
        a = st[k][:, 0] if st[k].dim() == 2 else st[k]
        a = a.detach().numpy()
        assert np.max(np.abs(a - ref)) <= 1e-10 * np.max(np.abs(ref)), k
    a1 = st["a"].detach().numpy()
    ra = np.stack([sim.arr["ax"], sim.arr["ay"], sim.arr["az"]], 1)
    assert np.max(np.abs(a1 - ra)) <= 1e-10 * np.max(np.abs(ra))
    assert abs(float(st["dt"]) - sim.dt) <= 1e-12 * sim.dt


def test_dense_gradients_match_central_differences():
    ic = _ic(250, 7)
    p = T.default_params(n_target=32.0, eos_mode=1, eps=0.01)
    st0 = T.state_from_ic(ic)
    probes = torch.arange(0, 250, 7)

    def run(x, v, u, K=2):
        st = dict(st0)
        st.update(x=x, v=v, u=u)
        for _ in range(K):
            st = T.step(st, p)
        return T.loss_ke_density(st, probes)

    x, v, u = (st0[k].clone().requires_grad_(True) for k in ("x", "v", "u"))
    run(x, v, u).backward()
    rs = np.random.default_rng(1)
    for name, g in (("x", x.grad), ("v", v.grad), ("u", u.grad)):
        base = st0[name]
        for _ in range(2):
            idx = tuple(int(rs.integers(0, s)) for s in base.shape)
            e = 1e-6 * max(abs(float(base[idx])), 1e-2)
            args = {"x": st0["x"], "v": st0["v"], "u": st0["u"]}
            bp, bm = base.clone(), base.clone()
            bp[idx] += e
            bm[idx] -= e
            with torch.no_grad():
                args[name] = bp
                lp = float(run(args["x"], args["v"], args["u"]))
                args[name] = bm
                lm = float(run(args["x"], args["v"], args["u"]))
            fd = (lp - lm) / (2 * e)
            scale = max(abs(fd), 1e-3 * float(g.abs().max()))
            assert abs(float(g[idx]) - fd) <= 2e-5 * scale, (name, idx, float(g[idx]), fd)
