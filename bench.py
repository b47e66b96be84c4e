#!/usr/bin/env python
"""Benchmark of the SPH + self-gravity step (one JSON line on stdout).

Workload (the configuration the headline metric is quoted on): N = 1,048,576
particles, two n = 1.5 polytropes of 524,288 particles each (M = R = G = 1),
centres 4R apart, approaching head on at relative speed 1.0; ideal gas +
radiation EOS with mu = 0.62; N_ngb = 64; Plummer softening eps = 0.002;
mixed precision (FP32 gravity pair terms on FP64 anchors, FP64 accumulation;
FP64 SPH pair terms, h solve, EOS root, integration and reductions; the FP32
SPH pair loops are an option whose error is reported too).  Seeded synthetic
data: the reference has no dataset.

A step is one whole time step of the pipeline (sort, predict, tree,
solve_range, find_ngb, density, pressure, hydro, gravity, diagnostics,
timestep, kick) with the state resident in HBM.  The state (~500 MB) is far
larger than L2, so no flush is needed between steps.

  value        particle-steps/s of the mixed step (device time, CUDA events,
               max over ranks)
  e2e          the same through the C ABI with host buffers: every step copies
               the state in from pinned host memory and the result out
  fp64         the plain FP64 step on the same workload, and the mixed/fp64
               ratio; errors = mixed vs FP64 accelerations at the same state,
               and (errors.against_oracle) every GPU form vs the FP64 oracle
  roofline     the direct-N gravity kernel on the FP32 FMA pipe: 20 flops per
               pair interaction x N^2 per launch / launch time, against the
               FP32 FMA peak measured in the same run
  adjoint      reverse sweep / forward step at the h solve's forward default
               and at the gradient tests' tolerance
  drift_100    energy drift over 100 steps, mixed and FP64 side by side
  dropin       the reference's own driver on this library (N = 262,144)
  large_c5     the N = 4,194,304 cold-sphere workload (5 mixed steps, tree
               gravity, a subset adjoint)
  cpu_baseline the FP64 oracle at this workload's own parameters on a bounded
               sample (see 'sample'; measured and extrapolated seconds are
               labelled), with the reference's own CPU build beside it
  c2_per_kernel the N = 262,144 FP64 workload, each kernel against its CPU
               counterparts

--impl reference times the reference's CPU build on the same workload (and
the oracle at the workload's parameters once).  Under torchrun (N > 1) the
ranks share ONE simulation of the same workload (cudasph_b200.sharded: SPH
leaf ranges and gravity work items per rank, an all-gather and two
all-reduces per step; strong scaling); rank 0 prints.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at N=1M, mixed vs FP64 at stated error; adjoint/forward cost"
UNIT = "particle-steps/s"


def workload_ic(n_total: int, seed: int = 12345 + 3):
    from cudasph_b200 import ics
    return ics.two_star_collision(n_total // 2, separation=4.0, rel_speed=1.0, n_poly=1.5, n_ngb=64.0, seed=seed,
                                  mu=0.62)


WORKLOAD_PARAMS = dict(n_target=64.0, eos_mode=1, soft_mode=1, eps=0.002)


def workload_name(n):
    return (f"two n=1.5 polytropes head-on (2 x {n // 2}), N={n}, gas+radiation EOS mu=0.62, N_ngb=64, "
            f"Plummer eps=0.002")


# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples during the timed region (every 200 ms)."""

    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return None
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 8:
                    continue
                if self.uuid and parts[0] != self.uuid:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[4:8]))
                except ValueError:
                    continue
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        sm = [r[0] for r in rows]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


def gpu_uuid():
    try:
        import torch
        u = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


# ----------------------------------------------------------------------------
def time_steps(sim, steps, warmup):
    """Device time of `steps` whole steps: CUDA events on the context's
    stream around them (the whole span, gaps between launches included),
    plus the per-phase device times for the breakdown."""
    import torch
    sim.step(warmup)
    sim.synchronize()
    sim.reset_counters()
    sim.set_profiling(True)
    st = sim.torch_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(st)
    sim.step(steps)
    e1.record(st)
    e1.synchronize()
    wall = time.perf_counter() - t0
    ph = sim.phase_times()
    sim.set_profiling(False)
    dev_ms = e0.elapsed_time(e1)
    return dev_ms, wall, ph, sim.kernel_launches()


def step_span_ms(sim, k=1):
    """CUDA-event span of k whole steps on the context's stream."""
    import torch
    st = sim.torch_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.step(k)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def rms_rel(a, b):
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1)) / np.mean(np.sum(b ** 2, axis=1))))


def traffic_from_profiles(kernel_tag: str, n: int):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary
    (profiles/<kernel_tag>.md, line 'traffic_bytes_per_launch_at_N=<n0>: <B>';
    for the mixed gravity kernel captured at the bench size itself, N = 1M),
    scaled to n in proportion to the particles when n differs: the 32-byte
    source records and the 32-byte output records the pair kernel accumulates
    into (64 MB at N = 1M) stay resident in L2 across the N^2 interactions,
    so DRAM sees each record about once per launch."""
    path = os.path.join(ROOT, "profiles", kernel_tag + ".md")
    if not os.path.exists(path):
        return None
    import re
    txt = open(path).read()
    m = re.search(r"traffic_bytes_per_launch_at_N=(\d+):\s*([0-9.eE+]+)", txt)
    if not m:
        return None
    n0, b0 = int(m.group(1)), float(m.group(2))
    return b0 * (n / n0)


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (no measured peaks file)"


# Algorithmic bytes per particle of the bandwidth-bound phases, each stream
# counted once; nbar = mean neighbour count.  Neighbour records gathered by the
# list loops (64-128 B per pair) are Morton-close and served by L1/L2; they
# are not part of the algorithmic figure.
SPH_BYTES = {
    # pos read 32; range 8, count 4 and the list 4 nbar written
    "solve_range": lambda nb: 32 + 8 + 4 + 4 * nb,
    # list 4 nbar + count 4 + own pos/vel 64 read; rho 8 + div/curl/omega/psi 32 written
    "density": lambda nb: 4 * nb + 4 + 64 + 40,
    # rho, P, u, mu 32 read; P 8 written
    "pressure": lambda nb: 40,
    # list 4 nbar + count 4 + own pos/vel/hyd/dd 128 read; dots 32 + vsig 8 written
    "hydro": lambda nb: 4 * nb + 4 + 128 + 40,
    # bounding box 32 + Morton keys (32 read, 12 written) + 8 radix passes x (12 read + 12 written)
    # + permutation of the state (204 read + 204 written + 4 index)
    "sort": lambda nb: 32 + 44 + 8 * 24 + 412,
}


# bytes of neighbour records each pair gathers (served by L1/L2): density
# reads pos + vel of j, hydro pos + vel + hyd + dd of j
# bytes gathered per pair: the neighbour's pos + vel (density); pos + vel +
# its per-particle factors {c, P / rho^2, Balsara} (hydro)
SPH_GATHER = {"density": 64, "hydro": 96}


def sph_bandwidth(ph, steps, n, nbar, l2_gbs=None):
    """Achieved HBM bandwidth of the bandwidth-bound phases (device time per
    step from the CUDA-event phase timers) against the measured copy peak,
    and the rate at which the pair loops gather neighbour records from L1/L2
    against the L2 read rate measured in the same run (cudasph_l2_peak; the
    pool's peaks file has no L2 figure).  L1 hits can lift a gather rate above
    the L2 figure."""
    peak, src = measured_hbm_gbs()
    out = {"peak_gbs": peak, "peak_source": src, "mean_neighbours": nbar}
    if l2_gbs:
        out["l2_read_gbs"] = round(l2_gbs, 1)
        out["l2_source"] = "L2 read probe in this run (48 MB resident buffer, 32-byte L2-only loads from every SM)"
    for k, f in SPH_BYTES.items():
        if k not in ph or ph[k][0] <= 0:
            continue
        ms = ph[k][0] / steps
        b = f(nbar) * n
        out[k] = {"ms": round(ms, 4), "bytes_per_particle": round(f(nbar), 1), "gbs": round(b / (ms * 1e-3) / 1e9, 1),
                  "frac": round(b / (ms * 1e-3) / 1e9 / peak, 4)}
        if k in SPH_GATHER:
            g = SPH_GATHER[k] * nbar * n / (ms * 1e-3) / 1e9
            out[k]["gather_gbs"] = round(g, 1)
            if l2_gbs:
                out[k]["gather_frac_of_l2"] = round(g / l2_gbs, 4)
    return out


ADJOINT_N = 65536
ADJOINT_PARAMS = dict(n_target=50.0, eos_mode=1, soft_mode=1, eps=0.01)


def adjoint_cost(steps=5, warmup=3, headline_n=None):
    """Cost of the hand-written adjoint of one step relative to the forward
    step, on the differentiation workload: an n=3 polytrope, N = 65,536,
    ideal gas + radiation EOS, N_ngb = 50, Plummer eps = 0.01.  Device time
    (CUDA events) of the forward step taken with keep on vs the reverse sweep
    (cudasph_adjoint) of the same step, each the median over `steps`
    step + adjoint iterations; a checkpointed rollout additionally replays
    each step once before its reverse sweep."""
    from cudasph_b200 import ics
    from cudasph_b200.simulation import Simulation, make_params
    ic = ics.polytrope(ADJOINT_N, n_poly=3.0, n_ngb=50.0, seed=12345 + 4, mu=0.62)
    out = {"workload": f"n=3 polytrope, N={ADJOINT_N}, gas+radiation EOS mu=0.62, N_ngb=50, Plummer eps=0.01"}
    def step_and_adjoint(sim, m):
        fwd = step_span_ms(sim)
        for k in ("vx", "vy", "vz"):
            sim.adjoint_set(k, m * sim.get(k))
        sim.adjoint()
        return fwd

    # the h solve at the reference's tolerance (rel_err 1e-3, 20 iterations: the
    # forward step's setting) and at the tight tolerance the gradient tests use
    # (rel_err 1e-12, 80 iterations), where the solved range is the root that
    # the adjoint's implicit derivative of the h solve describes
    settings = (("fp64", 0, 1e-3, 20), ("mixed", 1, 1e-3, 20),
                ("fp64_tight_h", 0, 1e-12, 80), ("mixed_tight_h", 1, 1e-12, 80))
    for name, prec, rel_err, max_iter in settings:
        sim = Simulation(ic, make_params(precision=prec, rel_err=rel_err, max_iter=max_iter, **ADJOINT_PARAMS))
        sim.set_keep(True)
        m = ic["m"]
        for _ in range(warmup):  # warm-up includes the reverse sweep (first use of its kernels)
            step_and_adjoint(sim, m)
        fwd_s, adj_s = [], []
        for _ in range(steps):
            sim.synchronize()
            sim.reset_counters()
            sim.set_profiling(True)
            fwd_s.append(step_and_adjoint(sim, m))
            ph = sim.phase_times()
            sim.set_profiling(False)
            adj_s.append(ph["adjoint"][0])
        fwd, adj = float(np.median(fwd_s)), float(np.median(adj_s))
        out[name] = {"rel_err": rel_err, "max_iter": max_iter, "forward_ms": fwd, "adjoint_ms": adj,
                     "adjoint_over_forward": adj / fwd,
                     "replay_plus_adjoint_over_forward": (fwd + adj) / fwd, "flags": sim.device_status(),
                     "samples_forward_ms": [round(v, 3) for v in fwd_s],
                     "samples_adjoint_ms": [round(v, 3) for v in adj_s]}
        sim.close()
    if headline_n:
        # the same ratio on the headline workload (mixed form, one step)
        ic = workload_ic(headline_n)
        sim = Simulation(ic, make_params(**dict(WORKLOAD_PARAMS, precision=1)))
        sim.set_keep(True)
        for _ in range(2):
            step_and_adjoint(sim, ic["m"])
        sim.synchronize()
        sim.reset_counters()
        sim.set_profiling(True)
        fwd = step_and_adjoint(sim, ic["m"])
        ph = sim.phase_times()
        sim.set_profiling(False)
        adj = ph["adjoint"][0]
        out["headline_workload_mixed"] = {"n": headline_n, "rel_err": 1e-3, "forward_ms": fwd, "adjoint_ms": adj,
                                          "adjoint_over_forward": adj / fwd,
                                          "replay_plus_adjoint_over_forward": (fwd + adj) / fwd,
                                          "flags": sim.device_status()}
        sim.close()
    return out


def tree_gravity(ic, thetas=(0.3, 0.5), reps=3, params=None, step_reps=3):
    """The opt-in Barnes-Hut gravity (grav_mode = tree, quadrupoles) on the
    same state as the headline: CUDA-event time of the gravity phase (radix
    tree + node moments + walk) per opening angle and its RMS force error
    against the direct mixed-precision sum (itself within 4e-8 of FP64 on
    this workload); then `step_reps` whole steps in that mode after one
    warm-up step (CUDA-event span on the context's stream), the throughput a
    run with tree gravity gets.  The direct sum stays the headline path."""
    from cudasph_b200.simulation import Simulation, make_params
    params = params or WORKLOAD_PARAMS
    d = Simulation(ic, make_params(**dict(params, precision=1)))
    d.CUDA_gravity()
    gd = np.stack([d.get(k) for k in ("gx", "gy", "gz")], 1)
    d.close()
    out = {}
    for th in thetas:
        s = Simulation(ic, make_params(**dict(params, precision=1, grav_mode=1, theta=th)))
        s.CUDA_gravity()  # sort + tree
        s.synchronize()
        s.reset_counters()
        s.set_profiling(True)
        for _ in range(reps):
            s.CUDA_gravity()
        ph = s.phase_times()
        s.set_profiling(False)
        g = np.stack([s.get(k) for k in ("gx", "gy", "gz")], 1)
        out[f"theta_{th}"] = {"ms": ph["gravity"][0] / reps, "rms_force_rel_vs_direct": rms_rel(g, gd),
                              "flags": s.device_status()}
        if step_reps > 0:
            s.step(1)
            s.synchronize()
            step_ms = step_span_ms(s, step_reps) / step_reps
            out[f"theta_{th}"].update(step_ms=step_ms, particle_steps_per_s=ic["x"].size / (step_ms * 1e-3),
                                      step_flags=s.device_status())
        s.close()
    return out


def energy_drift(n, steps):
    """Energy conservation over `steps` steps of the bench workload at N = n:
    the mixed form and the FP64 form run side by side from the same initial
    conditions (the FP64 GPU step equals the FP64 oracle to 1e-12 per kernel
    and 1e-8 over whole steps in the parity tests; the oracle itself cannot
    run N = 1M steps in bounded time).  Reported: each form's relative drift
    (E_K - E_0) / |E_0|, and the largest |E_mixed - E_fp64| / |E_0| over the
    run (same step index; the two forms' timesteps differ by rounding only).
    The energy is a by-product of each step's force pass, so E_0 is the energy
    after the first step and the K steps follow it."""
    import time
    from cudasph_b200.simulation import Simulation, make_params
    ic = workload_ic(n)
    res = {"workload": workload_name(n), "steps": steps}
    E = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        s = Simulation(ic, make_params(**dict(WORKLOAD_PARAMS, precision=prec)))
        e, t0 = [], time.perf_counter()
        s.step()
        e0 = s.system_statistics()["E"]
        for _ in range(steps):
            s.step()
            e.append(s.system_statistics()["E"])
        s.synchronize()
        E[name] = np.array(e)
        res[name] = {"E0": e0, "E_end": e[-1], "drift_rel": (e[-1] - e0) / abs(e0), "t_end": s.time,
                     "wall_s": time.perf_counter() - t0, "device_flags": s.device_status()}
        s.close()
    res["mixed_vs_fp64_max_rel"] = float(np.max(np.abs(E["mixed"] - E["fp64"])) / abs(res["fp64"]["E0"]))
    return res


LARGE_N = 1 << 22
LARGE_PARAMS = dict(n_target=50.0, eos_mode=0, soft_mode=1, eps=0.001)


def large_run(n=LARGE_N, steps=5, n_sub=262144):
    """The gravity-dominated workload: N = 4,194,304 cold uniform-density
    sphere (virial ratio 0.1, u = 1e-6, seeded positions), ideal gas,
    N_ngb = 50, Plummer eps = 0.001; `steps` mixed-precision steps (device
    time per phase, CUDA events; the first step solves h from the initial
    guess), gravity interactions/s against the FP32 FMA peak measured in the
    same run; then one adjoint step (gravity + hydro forces and the rest of
    the step) on a seeded 262,144-particle subset of the same sphere (masses
    scaled so the subset keeps the total mass)."""
    from cudasph_b200 import ics, _capi
    from cudasph_b200.simulation import Simulation, make_params
    L = _capi.lib()
    peak32 = L.cudasph_fma_peak(1, 4096, None)
    ic = ics.cold_sphere(n, virial=0.1, u0=1e-6, n_ngb=50.0, seed=12345 + 5)
    res = {"workload": f"cold uniform sphere, N={n}, virial 0.1, u=1e-6, ideal gas, N_ngb=50, Plummer eps=0.001, "
                       f"mixed precision", "steps": steps}
    sim = Simulation(ic, make_params(precision=1, **LARGE_PARAMS))
    sim.reset_counters()
    sim.set_profiling(True)
    step_ms = step_span_ms(sim, steps) / steps
    ph = sim.phase_times()
    sim.set_profiling(False)
    gms = ph["gravity"][0] / steps
    res["ms_per_step"] = step_ms
    res["particle_steps_per_s"] = n / (step_ms * 1e-3)
    res["phase_ms_per_step"] = {k: round(v[0] / steps, 3) for k, v in ph.items()}
    res["gravity"] = {"ms_per_launch": gms, "interactions_per_s": n * n / (gms * 1e-3),
                      "tflops_at_20_per_interaction": 20.0 * n * n / (gms * 1e-3) / 1e12,
                      "fp32_fma_peak_tflops": peak32 / 1e12,
                      "frac_of_fp32_peak": 20.0 * n * n / (gms * 1e-3) / peak32}
    res["stats_last_step"] = {k: v for k, v in sim.system_statistics().items() if k in ("E", "dt", "ngb_mean")}
    res["device_flags"] = sim.device_status()
    sim.close()
    # the opt-in tree gravity on the initial state, against the direct sum
    res["tree_gravity_initial_state"] = tree_gravity(ic, params=LARGE_PARAMS)

    rng = np.random.default_rng(12345 + 5)
    idx = np.sort(rng.choice(n, n_sub, replace=False))
    sub = {k: (np.asarray(v)[idx].copy() if isinstance(v, np.ndarray) else v) for k, v in ic.items()}
    sub["m"] = sub["m"] * (n / n_sub)
    rho = np.full(n_sub, 3.0 / (4.0 * math.pi))
    sub["range"] = ics.initial_range(rho, sub["m"], 50.0)
    s2 = Simulation(sub, make_params(precision=1, **LARGE_PARAMS))
    s2.set_keep(True)
    m = sub["m"]
    for _ in range(3):  # warm-up includes the reverse sweep
        s2.step()
        for k in ("vx", "vy", "vz"):
            s2.adjoint_set(k, m * s2.get(k))
        s2.adjoint()
    s2.synchronize()
    s2.reset_counters()
    s2.set_profiling(True)
    fwd = step_span_ms(s2)
    for k in ("vx", "vy", "vz"):
        s2.adjoint_set(k, m * s2.get(k))
    s2.adjoint()
    s2.synchronize()
    ph2 = s2.phase_times()
    s2.set_profiling(False)
    adj = ph2["adjoint"][0]
    res["adjoint_subset"] = {"n": n_sub, "forward_ms": fwd, "adjoint_ms": adj, "adjoint_over_forward": adj / fwd,
                             "loss": "kinetic energy after the step", "device_flags": s2.device_status()}
    s2.close()
    return res


C2_N = 262144
C2_PARAMS = dict(n_target=64.0, eos_mode=1, soft_mode=1, eps=0.005)


def c2_run(n=C2_N, steps=50, n_grav_targets=512):
    """The plain FP64 workload at N = 262,144 (n=1.5 polytrope with a seeded
    5 % perturbation of u, ideal gas + radiation EOS mu = 0.62, N_ngb = 64,
    Plummer eps = 0.005): `steps` FP64 steps on the GPU (device time per
    phase, CUDA events; energy change over the run), and the same phases on
    the CPU on the same initial state, each kernel against its CPU
    counterpart: the FP64 oracle restatement of the reference loops with the
    same parameters (OpenMP over all host threads; gravity on a seeded sample
    of targets extrapolated to n) and the reference's own code built for the
    host (its compiled-in DESIRED_NGB = 24 and spline softening)."""
    from cudasph_b200 import ics
    from cudasph_b200.simulation import Simulation, make_params
    from oracle import oracle as O
    ic = ics.polytrope(n, n_poly=1.5, n_ngb=64.0, seed=12345 + 2, u_jitter=0.05, mu=0.62)
    res = {"workload": f"n=1.5 polytrope, N={n}, u x (1 + U(-0.05, 0.05)), gas+radiation EOS mu=0.62, N_ngb=64, "
                       f"Plummer eps=0.005, FP64", "steps": steps}
    # GPU: the first step separately (h solved from the initial guess), then the run
    sim = Simulation(ic, make_params(precision=0, **C2_PARAMS))
    sim.reset_counters()
    sim.set_profiling(True)
    sim.step()
    sim.synchronize()
    first = sim.phase_times()
    sim.reset_counters()
    E0 = sim.system_statistics()["E"]
    sim.step(steps - 1)
    sim.synchronize()
    ph = sim.phase_times()
    sim.set_profiling(False)
    E1 = sim.system_statistics()["E"]
    gpu = {k: v[0] / (steps - 1) for k, v in ph.items() if v[1] > 0}
    res["gpu_ms_per_step"] = {k: round(v, 4) for k, v in gpu.items()}
    res["gpu_first_step_ms"] = {k: round(v[0], 4) for k, v in first.items() if v[1] > 0}
    res["energy_change_rel"] = (E1 - E0) / abs(E0)
    res["device_flags"] = sim.device_status()
    sim.close()
    # CPU: the FP64 oracle, phase by phase, on the initial state with the same parameters
    par = O.make_params(**C2_PARAMS)
    t = {}
    t0 = time.perf_counter()
    rng, _, _ = O.solve_range(ic["x"], ic["y"], ic["z"], ic["range"], par)
    t["solve_range"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    cnt, off, lst = O.find_ngb(ic["x"], ic["y"], ic["z"], rng)
    t["find_ngb"] = time.perf_counter() - t0
    st = dict(ic, range=rng)
    t0 = time.perf_counter()
    st.update(O.density(st, off, lst))
    t["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    st["P"] = O.pressure(st["rho"], st["u"], st["mu"], par)
    t["pressure"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.hydro(st, off, lst, par)
    t["hydro"] = time.perf_counter() - t0
    tg = np.random.default_rng(0).choice(n, size=n_grav_targets, replace=False).astype(np.int32)
    t0 = time.perf_counter()
    O.gravity(ic["x"], ic["y"], ic["z"], ic["m"], rng, par, targets=tg)
    t["gravity"] = (time.perf_counter() - t0) * n / n_grav_targets
    # the GPU's h solve writes the lists (find_ngb fused), so compare the pair
    cpu_ms = {k: 1000.0 * v for k, v in t.items()}
    gpu_solve = gpu.get("solve_range", 0.0) + gpu.get("find_ngb", 0.0)
    rows = {"solve_range + find_ngb": (cpu_ms["solve_range"] + cpu_ms["find_ngb"], gpu_solve)}
    for k in ("density", "pressure", "hydro", "gravity"):
        rows[k] = (cpu_ms[k], gpu.get(k, 0.0))
    res["per_kernel_vs_oracle_cpu"] = {
        k: {"cpu_ms": round(c, 2), "gpu_ms": round(g, 4), "speedup": round(c / g, 1) if g > 0 else None}
        for k, (c, g) in rows.items()}
    res["oracle_cpu_threads"] = O.num_threads()
    res["oracle_cpu_note"] = (f"FP64 oracle on the initial state, same parameters; gravity on {n_grav_targets} "
                              f"seeded targets x {n} sources, extrapolated")
    # the reference's own code built for the host, on the same state (its compiled-in parameters)
    if O.ref_available():
        r = O.RefPipeline(ic).time_step(n_grav_targets=256)
        res["reference_cpu_build_s"] = {k: round(v, 3) for k, v in r.items()}
        res["reference_cpu_threads"] = O.ref().ref_num_threads()
    return res


def dropin_run(n=C2_N, steps=3):
    """The drop-in path as a user of the reference gets it: the reference's own
    C++ driver (its CUDAsph_iterate.cpp, step.cpp, sph_accelerations.cpp,
    CUDA_calls.cpp, CUDA_gravity.cpp, ... compiled unmodified and linked
    against this library in place of the reference's host_calls.cu:
    oracle/_ref/CUDAsph_iterate_b200) on a restart file of an n-particle
    n=1.5 polytrope (u x (1 + U(-0.05, 0.05)), mu 0.62) for `steps` steps.
    The driver's own compiled-in parameters apply (DESIRED_NGB = 24, spline
    softening, gas + radiation EOS).  Reported: the per-iteration wall seconds
    the driver prints (step.cpp:137-145) and its phase lines: the host kd-tree
    (kd_tree.cpp:97-114), the device time of the two library calls, the host
    j-side scatter (sph_accelerations.cpp:104-115) and the gravity call
    (CUDA_gravity.cpp:3-71); the steady figure is the median of the
    iterations after the first (which creates the library's context)."""
    import re
    from cudasph_b200 import ics, state_io
    from cudasph_b200.simulation import Simulation, make_params
    drv = os.path.join(ROOT, "oracle", "_ref", "CUDAsph_iterate_b200")
    if not os.path.exists(drv):
        return {"unavailable": "oracle/_ref/CUDAsph_iterate_b200 is not built (needs the reference sources)"}
    ic = ics.polytrope(n, n_poly=1.5, n_ngb=24.0, seed=12345 + 2, u_jitter=0.05, mu=0.62)
    ic = {k: (v.astype(np.float32).astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in ic.items()}
    # the driver runs while its time is below t_end: the native step under the
    # driver's parameters gives the times after each step (the first has dt = 0)
    sim = Simulation(ic, make_params(n_target=24.0, eos_mode=1, soft_mode=0, use_psi=1))
    times = []
    for _ in range(steps):
        sim.step()
        times.append(sim.time)
    sim.close()
    t_end = 0.5 * (times[-2] + times[-1]) if steps >= 2 else 1e-12
    with tempfile.TemporaryDirectory() as d:
        hdr = state_io.default_header(n, t_end=t_end, dt_out=0.0, dt=0.0, global_time=0.0, iteration_number=0)
        state_io.write_state(os.path.join(d, "init.bin"), hdr, ic)
        t0 = time.perf_counter()
        r = subprocess.run([drv, "init.bin"], cwd=d, capture_output=True, text=True, timeout=900)
        wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"error": f"driver exit {r.returncode}", "stderr_tail": r.stderr[-500:]}
    err = r.stderr

    def grab(pat):
        return [float(v) for v in re.findall(pat, err, flags=re.S)]

    num = r"([0-9.eE+-]+)"
    it = grab(r"Iteration took " + num + " seconds")
    res = {"workload": f"n=1.5 polytrope, N={n}, reference driver parameters (DESIRED_NGB=24, spline softening, "
                       f"gas+radiation EOS mu=0.62)",
           "iterations": len(it), "iteration_s": [round(v, 4) for v in it], "process_wall_s": round(wall, 2),
           "phase_s": {"kd_tree_host": grab(r"building kd-tree \.\.\..*?done in " + num + " sec"),
                       "device_calls": grab(r"Device was used for " + num + " seconds"),
                       "sph_accelerations": grab(r"done SPH accelerations in " + num + " sec"),
                       "add_ngb_acc_host": grab(r"add_ngb_acc on the host \.\.\.\s+done in " + num + " sec"),
                       "gravity": grab(r"Computing gravity \.\.\.\s+done in " + num + " sec")}}
    steady = it[1:] if len(it) > 1 else it
    if steady:
        res["s_per_step"] = float(np.median(steady))
        res["particle_steps_per_s"] = n / res["s_per_step"]
    return res


FIRST_STEP_FIELDS = ("range", "rho", "divv", "curlv", "omega", "psi", "P", "ax", "ay", "az", "du", "vsig", "gx",
                     "gy", "gz", "phi")


def first_step_fields(sim, order):
    """The outputs of a step in tree order (slot s = original particle
    order[s]); after the first step from the initial conditions (dt = 0, so
    the predictor leaves x, v and u as they are) the forces in ax..az (hydro
    + gravity) belong to the initial state."""
    return {k: sim.get(k)[order] for k in FIRST_STEP_FIELDS}


def oracle_pass(ic, first, n_grav_targets=2048, seed=0):
    """The cpu_baseline leg: the FP64 oracle (oracle/sph_oracle.c, OpenMP over
    all host threads) runs the force evaluation of the first step on the
    workload's initial state with the workload's own parameters (N_ngb = 64,
    Plummer eps = 0.002, gas + radiation EOS), in the GPU's tree order, each
    phase timed: h solve from the same guesses, neighbour lists, density,
    EOS, hydro with the j-side scatter over all particles; gravity for a
    seeded sample of targets against all sources, extrapolated to all
    targets.  The lists and everything after them are taken at the FP64 GPU
    step's ranges, so the same pass is the checker of the GPU's first steps:
    errors of each GPU form against the oracle (density, EOS, hydro over all
    particles; gravity and total force over the sampled targets)."""
    from oracle import oracle as O
    n = ic["x"].size
    par = O.make_params(**WORKLOAD_PARAMS)
    order = first.get("order")
    if order is None:
        k, _ = O.morton_keys(ic["x"], ic["y"], ic["z"])
        order = O.sort_order(k)
    s = {k: np.ascontiguousarray(np.asarray(ic[k], np.float64)[order]) for k in
         ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu")}
    t = {}
    t0 = time.perf_counter()
    r_o, _, _ = O.solve_range(s["x"], s["y"], s["z"], s["range"], par)
    t["solve_range"] = time.perf_counter() - t0
    r_gpu = first["fp64"]["range"] if "fp64" in first else r_o
    t0 = time.perf_counter()
    cnt, off, lst = O.find_ngb(s["x"], s["y"], s["z"], r_gpu)
    t["find_ngb"] = time.perf_counter() - t0
    s["range"] = r_gpu
    t0 = time.perf_counter()
    s.update(O.density(s, off, lst))
    t["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    s["P"] = O.pressure(s["rho"], s["u"], s["mu"], par)
    t["pressure"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    h = O.hydro(s, off, lst, par)
    t["hydro"] = time.perf_counter() - t0
    tg = np.sort(np.random.default_rng(seed).choice(n, n_grav_targets, replace=False)).astype(np.int32)
    t0 = time.perf_counter()
    g = O.gravity(s["x"], s["y"], s["z"], s["m"], r_gpu, par, targets=tg)
    tgs = time.perf_counter() - t0
    measured = sum(t.values()) + tgs
    step_s = sum(t.values()) + tgs * n / n_grav_targets
    cb = {"value": n / step_s, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
          "config": "this workload's own parameters (N_ngb=64, Plummer eps=0.002, gas+radiation EOS mu=0.62)",
          "sample": (f"FP64 oracle (C restatement of the reference loops, OpenMP) on the same {n}-particle initial "
                     f"state: h solve, neighbour lists, density, EOS, hydro + j-side scatter over all {n} "
                     f"particles; gravity for {n_grav_targets} seeded targets x {n} sources"),
          "measured_s": round(measured, 3), "gravity_sample_s": round(tgs, 3), "gravity_targets": n_grav_targets,
          "extrapolated": True, "extrapolation": f"gravity x {n}/{n_grav_targets}",
          "s_per_step_extrapolated": round(step_s, 3), "phase_s": {k: round(v, 3) for k, v in t.items()}}
    against = {}
    if "fp64" not in first:
        return cb, against
    g3 = np.stack(g[:3], 1)
    h3 = np.stack([h["ax"], h["ay"], h["az"]], 1)
    for form, f in first.items():
        if form == "order":
            continue
        a = np.stack([f["ax"], f["ay"], f["az"]], 1)
        gg = np.stack([f["gx"], f["gy"], f["gz"]], 1)
        e = {"h_identical_frac": float(np.mean(f["range"] == r_o)),
             "max_rho_rel": float(np.max(np.abs(f["rho"] / s["rho"] - 1))),
             "max_P_rel": float(np.max(np.abs(f["P"] / s["P"] - 1))),
             "rms_hydro_rel": rms_rel(a - gg, h3),
             "rms_du_rel": float(np.sqrt(np.mean((f["du"] - h["du"]) ** 2) / max(np.mean(h["du"] ** 2), 1e-300))),
             "max_vsig_rel": float(np.max(np.abs(f["vsig"] / h["vsig"] - 1))),
             "rms_gravity_rel": rms_rel(gg[tg], g3),
             "max_phi_rel": float(np.max(np.abs(f["phi"][tg] / g[3] - 1))),
             "rms_force_rel": rms_rel(a[tg], h3[tg] + g3)}
        against[form] = e
    against["note"] = (f"first step from the initial state (dt = 0); density, EOS and hydro over all {n} "
                       f"particles at the FP64 GPU step's ranges, gravity and total force (hydro + gravity) over "
                       f"{n_grav_targets} seeded targets; h_identical_frac: the GPU's ranges against the "
                       f"oracle's own h solve")
    return cb, against


def cpu_reference_sample(ic, n_grav_targets=2048):
    from oracle import oracle as O
    if not O.ref_available():
        return None
    R = O.RefPipeline(ic)
    t = R.time_step(n_grav_targets=n_grav_targets)
    return t, O.ref().ref_num_threads()


def run_ours(args, rank, world):
    import torch
    from cudasph_b200.simulation import Simulation, make_params
    from cudasph_b200 import _capi

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    n = args.n
    ic = workload_ic(n)
    kw = dict(WORKLOAD_PARAMS)
    if args.fp64_only:
        kw["precision"] = 0
    else:
        kw["precision"] = 1

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # FMA-pipe peaks measured in this run (roofline denominators)
    L = _capi.lib()
    peak32 = L.cudasph_fma_peak(1, 4096, None)
    peak64 = L.cudasph_fma_peak(0, 1024, None)
    l2_gbs = L.cudasph_l2_peak(200, None) / 1e9

    # --- the mixed (headline) step -------------------------------------------------
    sim = Simulation(ic, make_params(**kw), device=dev)
    sim.step(args.warmup)
    sim.synchronize()
    barrier()
    with ClockSampler(gpu_uuid()) as clk:
        dev_ms, wall, ph, launches = time_steps(sim, args.steps, 0)
        barrier()
    clocks = clk.summary()
    flags = sim.device_status()
    ms_step = dev_ms / args.steps
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms_step], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    value = n * 1000.0 / ms_step
    stats = sim.system_statistics()
    gms, gl = ph["gravity"]
    grav_ms = gms / max(gl, 1)
    sim.close()

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f64" if args.fp64_only else "f32+f64", "data": "synthetic (seeded)",
           "config": {"workload": workload_name(n), "n_particles": n, "precision": "fp64" if args.fp64_only else
                      "mixed (FP32 gravity pair terms, FP64 SPH pair terms)", "l2": "state (~%.0f MB) larger than L2; no flush" % (n * 500 / 1e6),
                      "parallelism": "single GPU"},
           "gpu_launches": int(launches),
           "phase_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in ph.items()},
           "device_flags": flags}
    if clocks:
        out["clocks"] = clocks
    if rank != 0:
        return None

    flops = 20.0 * n * n
    prec_peak = peak64 if args.fp64_only else peak32
    achieved = flops / (grav_ms * 1e-3)
    tag = "gravity_fp64_plummer" if args.fp64_only else "gravity_mixed_plummer"
    out["roofline"] = {"kernel": tag, "bound": "fp64_pipe" if args.fp64_only else "fp32_pipe",
                       "achieved": achieved / 1e12, "peak": prec_peak / 1e12, "unit": "TFLOP/s",
                       "frac": achieved / prec_peak, "traffic": traffic_from_profiles(tag, n),
                       "peak_source": "FMA-chain probe measured in this run (the pool's measured-peaks file "
                                      "has HBM and bf16 tensor figures only)",
                       "flops_per_launch": flops, "launch_ms": grav_ms,
                       "interactions_per_s": n * n / (grav_ms * 1e-3)}
    out["stats_last_step"] = {k: stats[k] for k in ("E", "W", "T", "U", "dt", "ngb_mean", "ngb_min", "ngb_max")}
    out["sph_roofline"] = sph_bandwidth(ph, args.steps, n, stats["ngb_mean"], l2_gbs if l2_gbs > 0 else None)

    # --- FP64 comparison and errors ----------------------------------------------
    first = {}  # tree-order fields after the first step of each form (the oracle check below)
    if not args.fp64_only and args.fp64_steps > 0:
        kw64 = dict(kw, precision=0)
        s64 = Simulation(ic, make_params(**kw64), device=dev)
        s32 = Simulation(ic, make_params(**kw), device=dev)
        s64.step(1)
        s32.step(1)
        order = s64.order()
        first["order"] = order
        first["fp64"] = first_step_fields(s64, order)
        first["mixed"] = first_step_fields(s32, order)
        a64 = np.stack([s64.get(k) for k in ("ax", "ay", "az")], 1)
        a32 = np.stack([s32.get(k) for k in ("ax", "ay", "az")], 1)
        g64 = np.stack([s64.get(k) for k in ("gx", "gy", "gz")], 1)
        g32 = np.stack([s32.get(k) for k in ("gx", "gy", "gz")], 1)
        p64, p32 = s64.get("phi"), s32.get("phi")
        r64, r32 = s64.get("rho"), s32.get("rho")
        du64, du32 = s64.get("du"), s32.get("du")
        errors = {"rms_force_rel": rms_rel(a32, a64), "rms_gravity_rel": rms_rel(g32, g64),
                  "max_phi_rel": float(np.max(np.abs(p32 / p64 - 1))),
                  "max_rho_rel": float(np.max(np.abs(r32 / r64 - 1))),
                  "rms_du_rel": float(np.sqrt(np.mean((du32 - du64) ** 2) / max(np.mean(du64 ** 2), 1e-300))),
                  "rms_hydro_rel": rms_rel(a32 - g32, a64 - g64),
                  "rms_force_rel_to_gravity_scale": float(np.sqrt(np.mean(np.sum((a32 - a64) ** 2, 1))
                                                                  / np.mean(np.sum(g64 ** 2, 1)))),
                  "against": "FP64 GPU step at the same state, first step (errors against the FP64 oracle: "
                             "errors.against_oracle, from the cpu_baseline leg)"}
        s32.close()
        # the option with the density and hydro pair terms in FP32 as well
        s3 = Simulation(ic, make_params(**dict(kw, mixed_sph=3)), device=dev)
        s3.step(1)
        first["mixed_sph_3"] = first_step_fields(s3, order)
        a3 = np.stack([s3.get(k) for k in ("ax", "ay", "az")], 1)
        g3 = np.stack([s3.get(k) for k in ("gx", "gy", "gz")], 1)
        errors["mixed_sph_3"] = {"rms_force_rel": rms_rel(a3, a64), "rms_hydro_rel": rms_rel(a3 - g3, a64 - g64),
                                 "note": "density and hydro pair terms also in FP32 (~0.5 % faster step)"}
        s3.close()
        dms64, _, ph64, _ = time_steps(s64, args.fp64_steps, 1)
        ms64 = dms64 / args.fp64_steps
        g64ms = ph64["gravity"][0] / max(ph64["gravity"][1], 1)
        s64.close()
        out["fp64"] = {"value": n * 1000.0 / ms64, "ms_per_step": ms64, "steps": args.fp64_steps,
                       "gravity_ms": g64ms, "gravity_frac_of_fp64_peak": flops / (g64ms * 1e-3) / peak64}
        out["mixed_over_fp64"] = ms64 / ms_step
        out["errors"] = errors

    # --- the opt-in tree gravity on the same state -------------------------------------
    if args.tree:
        out["tree_gravity"] = tree_gravity(ic)

    # --- adjoint / forward cost (the differentiation form) --------------------------
    if args.adjoint:
        out["adjoint"] = adjoint_cost(headline_n=n)

    # --- end to end through the C ABI with host buffers ----------------------------
    if args.e2e_steps > 0:
        from cudasph_b200._capi import FIELDS
        ins = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu", "ax", "ay", "az", "du")
        outs = ins + ("rho", "P")
        sim = Simulation(ic, make_params(**kw), device=dev)
        sim.step(2)
        sim.synchronize()
        # two pinned host buffer sets; each step reads one and writes the other
        bufs = [{k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in outs} for _ in range(2)]
        for k in ins:
            bufs[0][k][:] = sim.get(k)
        sim.step_host({k: bufs[0][k] for k in ins}, bufs[1])  # warm
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            src, dst = bufs[(i + 1) % 2], bufs[i % 2]
            sim.step_host({k: src[k] for k in ins}, dst)
        e2e_s = time.perf_counter() - t0
        sim.close()
        out["e2e"] = {"value": n * args.e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * n * len(ins),
                      "d2h_bytes_per_step": 8 * n * len(outs), "steps": args.e2e_steps,
                      "api": "cudasph_step_host (C ABI), pinned host buffers, wall clock"}

    # --- energy drift over 100 steps (mixed and FP64 side by side) -----------------------
    if args.drift_line_steps > 0:
        out[f"drift_{args.drift_line_steps}"] = energy_drift(n, args.drift_line_steps)

    # --- the drop-in path: the reference's own driver on this library ---------------------
    if args.dropin_steps > 0:
        di = dropin_run(steps=args.dropin_steps)
        out["dropin"] = di
        if "s_per_step" in di:
            out["dropin_s_per_step"] = di["s_per_step"]

    # --- the other named workloads: C5 (N = 4M cold sphere, gravity-dominated) ---------
    if args.large_line:
        out["large_c5"] = large_run()

    # --- CPU baseline: the FP64 oracle at this workload's own parameters (and the ------
    # --- checker of the first steps above), the reference's own code beside it ---------
    if args.cpu_baseline:
        cb, against = oracle_pass(ic, first, n_grav_targets=args.cpu_grav_targets)
        r = cpu_reference_sample(ic, n_grav_targets=args.cpu_grav_targets)
        if r is not None:
            t, cores = r
            cb["reference_build"] = {
                "value": n / t["step"], "unit": UNIT, "cores": cores, "kind": "reference",
                "config": "reference compiled-in: DESIRED_NGB=24, spline softening (not this workload's "
                          "N_ngb=64 / Plummer eps=0.002; its sources are compiled unmodified)",
                "sample": (f"reference device code + kd-tree built for the CPU (oracle/_ref), one step on the "
                           f"same {n}-particle initial state: kd-tree build, solve_range, find_ngb, density, "
                           f"pressure, hydro + scatter over all particles, gravity for {args.cpu_grav_targets} "
                           f"sampled targets x {n} sources"),
                "measured_s": round(sum(v for k, v in t.items() if k not in ("step", "gravity")), 3),
                "gravity_sample_s": round(t["gravity_sample"], 3), "gravity_targets": args.cpu_grav_targets,
                "extrapolated": True, "extrapolation": f"gravity x {n}/{args.cpu_grav_targets}",
                "s_per_step_extrapolated": round(t["step"], 3),
                "phase_s": {k: round(v, 3) for k, v in t.items()}}
        out["cpu_baseline"] = cb
        if against and "errors" in out:
            out["errors"]["against_oracle"] = against
        # C2 (N = 262,144, plain FP64): each kernel on the GPU against its CPU
        # counterparts (the oracle at the workload's parameters, the
        # reference's own build at its compiled-in ones)
        if args.c2_line:
            out["c2_per_kernel"] = c2_run()
    return out


def run_sharded(args, rank, world):
    """N > 1 ranks under torchrun: ONE simulation of n particles sharded over
    the ranks (cudasph_b200.sharded: leaf ranges of the SPH loops and shares
    of the gravity work items per rank, an all-gather and two all-reduces per step), so
    the total work is fixed as N grows (strong scaling).  Device time: CUDA
    events on each rank's context stream around the timed steps (collectives
    included), max over ranks."""
    import torch
    import torch.distributed as dist
    from cudasph_b200 import _capi
    from cudasph_b200.sharded import ShardedSimulation
    from cudasph_b200.simulation import make_params

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    n = args.n
    ic = workload_ic(n)
    kw = dict(WORKLOAD_PARAMS, precision=0 if args.fp64_only else 1)
    L = _capi.lib()
    peak = L.cudasph_fma_peak(0 if args.fp64_only else 1, 1024 if args.fp64_only else 4096, None)

    sim = ShardedSimulation(ic, make_params(**kw), rank, world, device=dev)
    sim.step(args.warmup)
    sim.synchronize()
    dist.barrier()
    st = sim.torch_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.reset_counters()
    sim.set_profiling(True)
    with ClockSampler(gpu_uuid()) as clk:
        e0.record(st)
        sim.step(args.steps)
        e1.record(st)
        e1.synchronize()
        dist.barrier()
    clocks = clk.summary()
    ph = sim.phase_times()
    sim.set_profiling(False)
    launches = sim.kernel_launches()
    flags = sim.device_status()
    ms_local = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms_local], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item())
    gms, gl = ph["gravity"]
    grav_ms = gms / max(gl, 1)
    phase_sum = sum(v[0] for v in ph.values()) / args.steps

    # end to end through the public API with host buffers: every rank copies
    # the whole state in (its replica), steps, and copies the state out
    e2e = None
    if args.e2e_steps > 0:
        ins = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu", "ax", "ay", "az", "du")
        outs = ins + ("rho", "P")
        # two pinned host buffer sets; each step reads one and writes the other
        bufs = [{k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in outs} for _ in range(2)]
        for k in ins:
            bufs[0][k][:] = sim.get(k)
        dist.barrier()
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            src, dst = bufs[i % 2], bufs[(i + 1) % 2]
            sim.set_state_host({k: src[k] for k in ins})
            sim.step()
            sim.get_state_host(dst)
        wall = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
        dist.all_reduce(wall, op=dist.ReduceOp.MAX)
        e2e = {"value": n * args.e2e_steps / float(wall.item()), "unit": UNIT, "h2d_bytes_per_step": 8 * n * len(ins),
               "d2h_bytes_per_step": 8 * n * len(outs), "steps": args.e2e_steps,
               "api": "ShardedSimulation set_state_host / step / get_state_host (C ABI), pinned host buffers, "
                      "wall clock, max over ranks, per rank"}
    sim.close()
    if rank != 0:
        return None
    flops = 20.0 * n * n / world
    out = {"metric": METRIC, "value": n * 1000.0 / ms_step, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f64" if args.fp64_only else "f32+f64", "data": "synthetic (seeded)",
           "config": {"workload": workload_name(n), "n_particles": n,
                      "precision": "fp64" if args.fp64_only else "mixed (FP32 gravity pair terms, FP64 SPH pair terms)",
                      "l2": "state (~%.0f MB) larger than L2; no flush" % (n * 500 / 1e6),
                      "parallelism": f"shard{world}: SPH leaf ranges + gravity work items per rank, replicated "
                                     f"state, per step an all-gather (density exchange) and two all-reduces (NCCL)"},
           "gpu_launches": int(launches),
           "phase_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in ph.items()},
           "exchange_and_gaps_ms_per_step": round(ms_local - phase_sum, 4),
           "device_flags": flags,
           "roofline": {"kernel": "gravity_fp64_plummer" if args.fp64_only else "gravity_mixed_plummer",
                        "bound": "fp64_pipe" if args.fp64_only else "fp32_pipe",
                        "achieved": flops / (grav_ms * 1e-3) / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                        "frac": flops / (grav_ms * 1e-3) / peak,
                        "traffic": traffic_from_profiles("gravity_mixed_plummer", n) if not args.fp64_only else None,
                        "peak_source": "FMA-chain probe measured in this run", "flops_per_launch": flops,
                        "launch_ms": grav_ms, "note": "rank 0's share (1/N of the pairs)"}}
    if clocks:
        out["clocks"] = clocks
    if e2e:
        out["e2e"] = e2e
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU implementation of the path
    (its device loops and kd-tree compiled for the host, oracle/_ref), on the
    same initial state, each step a bounded sample: the whole SPH pass over
    all particles plus the gravity of args.cpu_grav_targets seeded targets,
    the gravity extrapolated to all targets.  The FP64 oracle at this
    workload's own parameters is timed once beside it (the reference's
    sources fix DESIRED_NGB = 24 and spline softening)."""
    if rank != 0:
        return None
    from oracle import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference built for the host CPU) is missing"}
    n = args.n
    ic = workload_ic(n)
    times, measured, grav_s = [], [], []
    t_wall = time.perf_counter()
    for i in range(args.warmup + args.steps):
        R = O.RefPipeline(ic)
        t = R.time_step(n_grav_targets=args.cpu_grav_targets, seed=i)
        if i >= args.warmup:
            times.append(t["step"])
            measured.append(sum(v for k, v in t.items() if k not in ("step", "gravity")))
            grav_s.append(t["gravity_sample"])
    wall = time.perf_counter() - t_wall
    ms = 1000.0 * float(np.mean(times))
    value = n * 1000.0 / ms
    cores = O.ref().ref_num_threads()
    same_cfg, _ = oracle_pass(ic, {}, n_grav_targets=args.cpu_grav_targets)
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": workload_name(n), "n_particles": n,
                       "precision": "reference FP32 + float-float",
                       "reference_parameters": "compiled-in DESIRED_NGB=24 and spline softening"},
            "timing": {"ms_per_step": "extrapolated: measured SPH pass + gravity sample x N/targets",
                       "measured_s_per_step": round(float(np.mean(measured)) + float(np.mean(grav_s)), 3),
                       "gravity_sample_s": round(float(np.mean(grav_s)), 3),
                       "gravity_targets": args.cpu_grav_targets, "extrapolated": True,
                       "wall_s_all_steps": round(wall, 1)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"per step: full SPH pass over {n} particles with the reference's code "
                                       f"(DESIRED_NGB=24, spline softening), gravity on {args.cpu_grav_targets} "
                                       f"sampled targets x {n} sources extrapolated"},
            "oracle_same_config": same_cfg,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _json_stdout():
    """The JSON line goes to the process's original stdout; everything else
    written to file descriptor 1 from here on (libraries such as NCCL print
    their version there at communicator init, the reference's CPU code prints
    tree statistics) is sent to stderr, so stdout carries one JSON line."""
    out = os.fdopen(os.dup(1), "w")
    sys.stdout.flush()
    os.dup2(2, 1)
    return out


def main():
    json_out = _json_stdout()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--fp64-only", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=3)
    # gravity targets of the CPU baseline's bounded sample: with the SPH pass over
    # all particles, about 6 s of CPU work per sampled step at N = 1M on 16 threads
    ap.add_argument("--cpu-grav-targets", type=int, default=2048)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--drift-line-steps", type=int, default=100,
                    help="energy drift over this many steps of the mixed and FP64 forms in the bench line (0: skip)")
    ap.add_argument("--no-large-line", dest="large_line", action="store_false",
                    help="skip the N = 4,194,304 cold-sphere run (C5) in the bench line")
    ap.add_argument("--no-c2-line", dest="c2_line", action="store_false",
                    help="skip the N = 262,144 per-kernel GPU / CPU table (C2) in the bench line")
    ap.add_argument("--dropin-steps", type=int, default=3,
                    help="steps of the reference's own driver on this library (N = 262,144; 0: skip)")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false")
    ap.add_argument("--no-tree", dest="tree", action="store_false",
                    help="skip the tree-gravity measurement (opt-in Barnes-Hut mode)")
    ap.add_argument("--sharded", action="store_true",
                    help="run the sharded multi-GPU path also at N = 1 (a one-rank NCCL process group)")
    ap.add_argument("--drift-steps", type=int, default=0,
                    help="instead of the bench line, measure energy drift over this many steps (mixed vs FP64)")
    ap.add_argument("--c2", action="store_true",
                    help="instead of the bench line, run the N = 262,144 plain FP64 workload (50 steps) with each "
                         "kernel timed against its CPU counterpart")
    ap.add_argument("--large", action="store_true",
                    help="instead of the bench line, run the N = 4,194,304 cold-sphere workload (5 steps + a subset "
                         "adjoint)")
    args = ap.parse_args()
    if args.large:
        print(json.dumps({"measurement": "large_cold_sphere", **large_run()}), file=json_out, flush=True)
        return
    if args.c2:
        print(json.dumps({"measurement": "fp64_262k_per_kernel", **c2_run()}), file=json_out, flush=True)
        return
    if args.drift_steps > 0:
        print(json.dumps({"measurement": "energy_drift", **energy_drift(args.n, args.drift_steps)}), file=json_out,
              flush=True)
        return
    assert args.warmup >= 3 or args.impl == "reference" or os.environ.get("BENCH_ALLOW_SHORT_WARMUP")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    sharded = args.impl == "ours" and (world > 1 or args.sharded)
    if sharded:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(local)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29511")
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    try:
        if args.impl != "ours":
            out = run_reference(args, rank, world)
        elif sharded:
            out = run_sharded(args, rank, world)
        else:
            out = run_ours(args, rank, world)
    finally:
        if sharded:
            import torch.distributed as dist
            dist.destroy_process_group()
    if out is not None and rank == 0:
        print(json.dumps(out), file=json_out, flush=True)


if __name__ == "__main__":
    main()
