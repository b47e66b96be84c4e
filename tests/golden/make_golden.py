"""Generate the golden fixtures from the reference itself.

The reference ships no tests, fixtures or input data.  This script runs the
reference's own per-particle device code and host kd-tree, built for the CPU
from the reference sources by ``make -C oracle ref`` (oracle/_ref/
libref_cpu.so), on seeded synthetic inputs, and stores inputs and outputs:

  ref_tables.npz           kernel functions on a u grid (dev_sph_kernels.cu),
                           EOS pressures (dev_compute_pressure.cu), quartic
                           roots, Peano-Hilbert keys (sort_bodies.cpp:66-105)
  ref_pipeline_n2048.npz   one sph_accelerations + gravity pass on a 2048-
                           particle n=1.5 polytrope with a rotating, noisy
                           velocity field: solve_range, find_ngb CSR, density,
                           pressure, hydro (+ j-side scatter), gravity

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cudasph_b200 import ics  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tables():
    R = O.ref()
    u = np.linspace(0.0, 2.2, 441).astype(np.float32)
    k = {}
    for name, idx in O.KERNELS.items():
        out = np.zeros(u.size, np.float32)
        R.ref_kernel_eval(idx, u.size, u, out)
        k["k_" + name] = out
    rs = np.random.default_rng(2024)
    rho = (10 ** rs.uniform(-4, 2, 400)).astype(np.float32)
    uu = (10 ** rs.uniform(-3, 1, 400)).astype(np.float32)
    mu = rs.uniform(0.5, 1.4, 400).astype(np.float32)
    P = np.zeros(400, np.float32)
    R.ref_pressure(400, rho, uu, mu, P)
    ph_in = rs.integers(0, 1 << 18, size=(200, 3)).astype(np.int32)
    ph = np.array([R.ref_peano_key(int(a), int(b), int(c), 18) for a, b, c in ph_in], np.int64)
    np.savez_compressed(os.path.join(OUT, "ref_tables.npz"), u=u, eos_rho=rho, eos_u=uu, eos_mu=mu, eos_P=P,
                        ph_in=ph_in, ph_key=ph, **k)


def pipeline():
    n = 2048
    ic = ics.polytrope(n, n_ngb=24, seed=21)
    rs = np.random.default_rng(22)
    ic["vx"] = -0.3 * ic["y"] + rs.normal(0, 0.05, n)
    ic["vy"] = 0.3 * ic["x"] + rs.normal(0, 0.05, n)
    ic["vz"] = rs.normal(0, 0.05, n)
    P = O.RefPipeline(ic)
    inp = {k: P.pos[:, c].copy() for c, k in enumerate(("x", "y", "z", "range0"))}
    inp.update({k: P.vel[:, c].copy() for c, k in enumerate(("vx", "vy", "vz", "m"))})
    inp["u"] = P.hydro[:, 2].copy()
    inp["mu"] = P.hydro[:, 3].copy()
    P.kdtree()
    rng, nn_solve = P.solve_range(1e-3)
    cnt, off, lst = P.find_ngb()
    rho, dd = P.density()
    pres = P.pressure()
    dots, vsig = P.hydro_dots(1.0, 2.0)
    grav = P.gravity()
    np.savez_compressed(os.path.join(OUT, "ref_pipeline_n2048.npz"), **inp, range=rng, n_ngb_solve=nn_solve,
                        n_ngb=cnt, offsets=off, ngb_list=lst, rho=rho, divv=dd[:, 0], curlv=dd[:, 1],
                        omega=dd[:, 2], psi=dd[:, 3], P=pres, ax=dots[:, 0], ay=dots[:, 1], az=dots[:, 2],
                        du=dots[:, 3], vsig=vsig, gx=grav[:, 0], gy=grav[:, 1], gz=grav[:, 2], phi=grav[:, 3])


if __name__ == "__main__":
    tables()
    pipeline()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
