"""torch.autograd.Function over K steps of the device-resident step.

Forward runs K whole steps through the C ABI and keeps a checkpoint of the
particle state every `every` steps.  Backward walks the segments from the
last to the first: it re-runs the segment from its checkpoint to recover the
pre-step state of every step in it, then for each step (last first) replays
that one step with keep on and calls the hand-written adjoint kernels
(cudasph_adjoint), chaining the state adjoints from step to step.

Inputs:  x0 (N,3), v0 (N,3), u0 (N) -- float64 tensors (any device)
Outputs: v_K (N,3), rho_K (N) -- the velocities after K steps and the density
         computed in the last step; a loss such as kinetic energy plus the mean
         density at probe particles is formed from them in torch.
Gradients flow to x0, v0, u0.  This is a test / harness binding: the step and
its adjoint run in libcudasph_b200.so.
"""
from __future__ import annotations

import numpy as np
import torch

from .simulation import Simulation

STATE = ("x", "y", "z", "range", "vx", "vy", "vz", "u", "ax", "ay", "az", "du")


class RolloutContext:
    """The simulation and the fixed part of the initial conditions."""

    def __init__(self, ic: dict, params, steps: int, every: int = 5, device: int = 0):
        self.ic = ic
        self.params = params
        self.steps = int(steps)
        self.every = max(1, int(every))
        self.sim = Simulation(ic, params, device=device)
        self.sim.set_keep(True)

    def close(self):
        self.sim.close()

    def _set(self, st: dict):
        s = self.sim
        for k in STATE:
            s.set(k, st[k])
        s.set_time(st["time"], st["dt"])

    def _get(self) -> dict:
        s = self.sim
        out = {k: s.get(k) for k in STATE}
        out["time"], out["dt"] = s.time, s.dt
        return out


def _np(t):
    return t.detach().to("cpu", torch.float64).numpy()


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, u0, rc: RolloutContext):
        st = {k: np.asarray(rc.ic[k], np.float64).copy() for k in ("range", "ax", "ay", "az", "du")
              if k in rc.ic}
        n = x0.shape[0]
        for k in ("ax", "ay", "az", "du"):
            st.setdefault(k, np.zeros(n))
        xx, vv, uu = _np(x0), _np(v0), _np(u0)
        st.update(x=xx[:, 0].copy(), y=xx[:, 1].copy(), z=xx[:, 2].copy(), vx=vv[:, 0].copy(), vy=vv[:, 1].copy(),
                  vz=vv[:, 2].copy(), u=uu.copy(), time=float(rc.ic.get("time", 0.0)), dt=float(rc.ic.get("dt", 0.0)))
        rc._set(st)
        ckpt = {0: rc._get()}
        for s in range(rc.steps):
            rc.sim.step()
            if (s + 1) % rc.every == 0 and s + 1 < rc.steps:
                ckpt[s + 1] = rc._get()
        vK = np.stack([rc.sim.get(k) for k in ("vx", "vy", "vz")], 1)
        rhoK = rc.sim.get("rho")
        ctx.rc = rc
        ctx.ckpt = ckpt
        ctx.dev = x0.device
        return (torch.as_tensor(vK, device=x0.device), torch.as_tensor(rhoK, device=x0.device))

    @staticmethod
    def backward(ctx, gv, grho):
        rc, ckpt = ctx.rc, ctx.ckpt
        sim = rc.sim
        n = sim.n
        adj = {k: np.zeros(n) for k in ("x", "y", "z", "vx", "vy", "vz", "u", "ax", "ay", "az", "du")}
        if gv is not None:
            g = _np(gv)
            adj["vx"], adj["vy"], adj["vz"] = g[:, 0].copy(), g[:, 1].copy(), g[:, 2].copy()
        rho_bar = _np(grho) if grho is not None else None
        dtbar = 0.0
        starts = sorted(ckpt)
        for si in range(len(starts) - 1, -1, -1):
            s0 = starts[si]
            s1 = starts[si + 1] if si + 1 < len(starts) else rc.steps
            # pre-step states of the segment
            pre = [ckpt[s0]]
            rc._set(ckpt[s0])
            for s in range(s0, s1 - 1):
                sim.step()
                pre.append(rc._get())
            for s in range(s1 - 1, s0 - 1, -1):
                rc._set(pre[s - s0])
                sim.step()  # replays step s with keep on
                for k, v in adj.items():
                    sim.adjoint_set(k, v)
                if s == rc.steps - 1 and rho_bar is not None:
                    sim.adjoint_set("rho", rho_bar)
                sim.adjoint_set_dt(dtbar)
                sim.adjoint()
                for k in adj:
                    adj[k] = sim.adjoint_get(k)
                dtbar = sim.adjoint_get_dt()
        dev = ctx.dev
        gx = torch.as_tensor(np.stack([adj["x"], adj["y"], adj["z"]], 1), device=dev)
        gvv = torch.as_tensor(np.stack([adj["vx"], adj["vy"], adj["vz"]], 1), device=dev)
        gu = torch.as_tensor(adj["u"], device=dev)
        return gx, gvv, gu, None


def rollout(x0, v0, u0, rc: RolloutContext):
    return Rollout.apply(x0, v0, u0, rc)
