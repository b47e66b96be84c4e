"""The native C ABI driven from C++ with no Python in the loop
(tests/native_step.cpp, compiled here with g++ against the in-tree
library): three FP64 steps of a 4,096-particle polytrope must match the same
steps through the Python handle on the same library (to the rounding of the
FP64 atomics, whose order varies between runs)."""
import os
import subprocess

import numpy as np
import pytest

from cudasph_b200 import ics

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IN_FIELDS = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "u", "mu")


def test_cpp_program_on_the_native_abi(tmp_path):
    from cudasph_b200._capi import FIELDS, LIB_PATH
    from cudasph_b200.simulation import Simulation, make_params
    exe = tmp_path / "native_step"
    libdir = os.path.dirname(LIB_PATH)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native_step.cpp"), "-o", str(exe), "-L", libdir,
                    "-Wl,-rpath," + libdir, "-lcudasph_b200"], check=True)
    n = 4096
    ic = ics.polytrope(n, n_ngb=50, seed=23)
    rs = np.random.default_rng(23)
    for k in ("vx", "vy", "vz"):
        ic[k] = rs.normal(0, 0.05, n)
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([n], np.int32).tofile(f)
        for k in IN_FIELDS:
            np.ascontiguousarray(ic[k], np.float64).tofile(f)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "3"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    energies = [float(line.split()[3]) for line in r.stdout.splitlines() if line.startswith("step")]
    assert len(energies) == 3
    got = np.fromfile(tmp_path / "out.bin", np.float64).reshape(len(FIELDS), n)
    sim = Simulation(ic, make_params(n_target=50.0, eos_mode=0, soft_mode=1, eps=0.01, precision=0))
    for _ in range(3):
        sim.step()
    E = sim.system_statistics()["E"]
    assert abs(energies[-1] - E) <= 1e-12 * abs(E)
    for k in ("x", "vx", "u", "range", "rho", "ax", "phi"):
        a, b = got[FIELDS.index(k)], sim.get(k)
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), k
    sim.close()
