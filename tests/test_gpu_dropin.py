"""Drop-in: the reference's own C++ driver, unmodified, on this library.

oracle/_ref/CUDAsph_iterate_b200 is the reference's CUDAsph_iterate.cpp and
member-function sources (step.cpp, sph_accelerations.cpp, CUDA_calls.cpp,
CUDA_gravity.cpp, read/write_state.cpp, ...) compiled where they lie and
linked against libcudasph_b200.so instead of the reference's host_calls.cu
(oracle/Makefile, target 'driver').  The test writes a restart file, lets the
driver run two steps (the driver keeps float4 state on the host and scatters
the j-side pair force itself, sph_accelerations.cpp:106-114), reads its
restart.bin and compares with the native FP64 step under the reference's
parameters (DESIRED_NGB 24, spline softening, gas + radiation EOS).
"""
import os
import subprocess

import numpy as np
import pytest

from cudasph_b200 import ics, state_io

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "CUDAsph_iterate_b200")


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="reference driver not built (make -C oracle driver)")
def test_reference_driver_runs_on_this_library(tmp_path):
    from cudasph_b200.simulation import Simulation, make_params
    n = 4096
    ic = ics.polytrope(n, n_ngb=24, seed=17)
    ic = {k: (v.astype(np.float32).astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in ic.items()}
    hdr = state_io.default_header(n, t_end=1e-12, dt_out=0.0, dt=0.0, global_time=0.0, iteration_number=0)
    state_io.write_state(str(tmp_path / "init.bin"), hdr, ic)
    r = subprocess.run([DRIVER, "init.bin"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "end-of-simulation" in r.stderr
    lines = [ln.split() for ln in r.stdout.strip().splitlines()]
    assert len(lines) == 2  # two steps (t_end reached after the first dt > 0)
    h, p = state_io.read_state(str(tmp_path / "restart.bin"))

    sim = Simulation(ic, make_params(n_target=24.0, eos_mode=1, soft_mode=0, use_psi=1))
    sim.step()
    st1 = sim.system_statistics()
    sim.step()
    st2 = sim.system_statistics()

    def close(a, b, tol):
        return np.max(np.abs(a - b)) <= tol * np.max(np.abs(b))

    for k, tol in (("x", 1e-6), ("y", 1e-6), ("z", 1e-6), ("range", 2e-5), ("rho", 5e-4), ("u", 1e-5)):
        assert close(p[k], sim.get(k), tol), k
    v_ref = np.stack([p["vx"], p["vy"], p["vz"]], 1)
    v_nat = np.stack([sim.get(k) for k in ("vx", "vy", "vz")], 1)
    assert np.sqrt(np.mean(np.sum((v_ref - v_nat) ** 2, 1)) / np.mean(np.sum(v_nat ** 2, 1))) < 1e-3
    # the driver's per-step energy line (system_statistics.cpp:80-81: t W T U E S |J|)
    for line, st in zip(lines, (st1, st2)):
        t, W, T, U, E = (float(v) for v in line[:5])
        assert abs(W - st["W"]) <= 1e-4 * abs(st["W"])
        assert abs(U - st["U"]) <= 1e-4 * abs(st["U"])
        assert abs(E - st["E"]) <= 1e-3 * abs(st["E"])
    sim.close()


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="reference driver not built (make -C oracle driver)")
def test_reference_sort_order_equals_peano_key_mode(tmp_path):
    """The driver Peano-Hilbert sorts every 100th iteration (step.cpp:26-31,
    sort_bodies.cpp:119-186); a restart file at iteration 99 makes its first
    step sort, so its restart.bin holds the particles in the reference's own
    order.  That order must be the one the native context sorts into with
    key_mode = Peano-Hilbert (distinct keys, so the reference's qsort has no
    ties to order)."""
    from cudasph_b200.simulation import Simulation, make_params
    from oracle import oracle as O
    n = 4096
    ic = ics.polytrope(n, n_ngb=24, seed=23)
    ic = {k: (v.astype(np.float32).astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in ic.items()}
    k, _ = O.peano_keys(ic["x"], ic["y"], ic["z"])
    assert np.unique(k).size == n
    hdr = state_io.default_header(n, t_end=1e-12, dt_out=0.0, dt=0.0, global_time=0.0, iteration_number=99)
    state_io.write_state(str(tmp_path / "init.bin"), hdr, ic)
    r = subprocess.run([DRIVER, "init.bin"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Peano-Hilbert sorting" in r.stderr
    _, p = state_io.read_state(str(tmp_path / "restart.bin"))
    sim = Simulation(ic, make_params(n_target=24.0, eos_mode=1, soft_mode=0, use_psi=1, key_mode=1))
    sim.sort_bodies()
    order = sim.order()
    assert np.array_equal(order, O.sort_order(k))
    sim.step()
    sim.step()  # the driver's two steps; its restart.bin lists the particles in its sorted order
    for c, tol in (("x", 1e-6), ("y", 1e-6), ("z", 1e-6), ("u", 1e-5)):
        got = sim.get(c)[order]
        assert np.max(np.abs(p[c] - got)) <= tol * np.max(np.abs(got)), c
    sim.close()

