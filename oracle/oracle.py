"""ctypes binding of the FP64 CPU oracle (sph_oracle.c) and of the reference
built for the host CPU (ref_cpu_harness.cpp -> _ref/libref_cpu.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py.  The product (cudasph_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_cpu.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

KERNELS = {"w": 0, "dw": 1, "dwdh": 2, "dphidh": 3, "iw": 4, "ig": 5, "dig": 6, "digdh": 7, "diw": 8}


class OrcParams(C.Structure):
    _fields_ = [
        ("n_target", C.c_double), ("rel_err", C.c_double), ("max_iter", C.c_int), ("f_scale", C.c_double),
        ("av_alpha", C.c_double), ("av_beta", C.c_double), ("gamma", C.c_double), ("eos_mode", C.c_int),
        ("soft_mode", C.c_int), ("eps", C.c_double), ("use_psi", C.c_int), ("cn1", C.c_double),
        ("cn2", C.c_double), ("G", C.c_double),
    ]


def make_params(**kw) -> OrcParams:
    """Parameters with the reference's defaults (DESIRED_NGB 24, rel_err 1e-3,
    MAX_ITER 20, f_scale 0.1, alpha 1, beta 2, gamma 5/3, ideal+radiation EOS,
    spline softening, Courant 0.3/0.2, G = 1)."""
    d = dict(n_target=24.0, rel_err=1e-3, max_iter=20, f_scale=0.1, av_alpha=1.0, av_beta=2.0,
             gamma=5.0 / 3.0, eos_mode=1, soft_mode=0, eps=0.0, use_psi=None, cn1=0.3, cn2=0.2, G=1.0)
    d.update(kw)
    if d["use_psi"] is None:
        d["use_psi"] = 1 if d["soft_mode"] == 0 else 0
    return OrcParams(**d)


class OrcState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(k, C.POINTER(C.c_double)) for k in (
        "x", "y", "z", "range", "vx", "vy", "vz", "m", "rho", "P", "u", "mu",
        "divv", "curlv", "omega", "psi", "ax", "ay", "az", "du", "gx", "gy", "gz", "phi", "vsig")] + [
        ("n_ngb", C.POINTER(C.c_int)), ("dt", C.c_double), ("time", C.c_double), ("iteration", C.c_int),
        ("stats", C.c_double * 16)]


_lib = None
_ref = None


def _build(target: str):
    subprocess.run(["make", "-C", HERE, target], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        _build("all")
    L = C.CDLL(LIB_PATH)
    L.orc_kernel_eval.argtypes = [C.c_int, C.c_int, _dp, _dp]
    L.orc_solve_range.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _ip, _ip, C.POINTER(OrcParams)]
    L.orc_find_ngb.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _ip, _lp, C.c_void_p]
    L.orc_find_ngb.restype = C.c_longlong
    L.orc_density.argtypes = [C.c_int] + [_dp] * 8 + [_lp, _ip] + [_dp] * 5
    L.orc_pressure.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.POINTER(OrcParams)]
    L.orc_pressure_one.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(OrcParams)]
    L.orc_pressure_one.restype = C.c_double
    L.orc_quartic_root.argtypes = [C.c_double, C.c_double]
    L.orc_quartic_root.restype = C.c_double
    L.orc_hydro.argtypes = [C.c_int] + [_dp] * 14 + [_lp, _ip] + [_dp] * 5 + [C.c_void_p, C.POINTER(OrcParams)]
    L.orc_gravity.argtypes = [C.c_int, C.c_void_p, C.c_int] + [_dp] * 9 + [C.POINTER(OrcParams)]
    L.orc_gravity_src.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int] + [_dp] * 9 + [C.POINTER(OrcParams)]
    L.orc_solve_range_tgt.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                      C.POINTER(OrcParams)]
    L.orc_find_ngb_tgt.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp, _ip, _lp, C.c_void_p]
    L.orc_find_ngb_tgt.restype = C.c_longlong
    L.orc_density_tgt.argtypes = [C.c_int, _ip] + [_dp] * 8 + [_lp, _ip] + [_dp] * 5
    L.orc_hydro_tgt.argtypes = [C.c_int, _ip, C.c_int] + [_dp] * 14 + [_dp] * 5 + [C.POINTER(OrcParams)]
    L.orc_morton_keys.argtypes = [C.c_int, _dp, _dp, _dp, _up, C.c_void_p]
    L.orc_peano_keys.argtypes = [C.c_int, _dp, _dp, _dp, _up, C.c_void_p]
    L.orc_peano_hilbert_key.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.orc_peano_hilbert_key.restype = C.c_uint64
    L.orc_sort_order.argtypes = [C.c_int, _up, _ip]
    L.orc_timestep.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.POINTER(OrcParams)]
    L.orc_timestep.restype = C.c_double
    L.orc_step.argtypes = [C.POINTER(OrcState), C.POINTER(OrcParams)]
    L.orc_statistics.argtypes = [C.POINTER(OrcState), _dp]
    L.orc_num_threads.restype = C.c_int
    _lib = L
    return L


def num_threads() -> int:
    return lib().orc_num_threads()


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def kernel_eval(name: str, u) -> np.ndarray:
    u = _f64(u)
    out = np.empty_like(u)
    lib().orc_kernel_eval(KERNELS[name], u.size, u, out)
    return out


def solve_range(x, y, z, range0, params: OrcParams):
    x, y, z = _f64(x), _f64(y), _f64(z)
    rng = _f64(range0).copy()
    n = x.size
    nn = np.zeros(n, np.int32)
    ne = np.zeros(n, np.int32)
    lib().orc_solve_range(n, x, y, z, rng, nn, ne, C.byref(params))
    return rng, nn, ne


def find_ngb(x, y, z, rng):
    """Exact neighbour lists {j : ds2 < range_i^2} (ascending j) as CSR."""
    x, y, z, rng = _f64(x), _f64(y), _f64(z), _f64(rng)
    n = x.size
    cnt = np.zeros(n, np.int32)
    off = np.zeros(n + 1, np.int64)
    tot = lib().orc_find_ngb(n, x, y, z, rng, cnt, off, None)
    lst = np.zeros(max(tot, 1), np.int32)
    lib().orc_find_ngb(n, x, y, z, rng, cnt, off, lst.ctypes.data_as(C.c_void_p))
    return cnt, off, lst[:tot]


def density(s: dict, off, lst):
    n = s["x"].size
    out = {k: np.zeros(n) for k in ("rho", "divv", "curlv", "omega", "psi")}
    lib().orc_density(n, *[_f64(s[k]) for k in ("x", "y", "z", "range", "vx", "vy", "vz", "m")],
                      np.ascontiguousarray(off, np.int64), np.ascontiguousarray(lst, np.int32),
                      out["rho"], out["divv"], out["curlv"], out["omega"], out["psi"])
    return out


def pressure(rho, u, mu, params: OrcParams):
    rho, u, mu = _f64(rho), _f64(u), _f64(mu)
    P = np.zeros_like(rho)
    lib().orc_pressure(rho.size, rho, u, mu, P, C.byref(params))
    return P


def quartic_root(q: float, r: float) -> float:
    return lib().orc_quartic_root(q, r)


def hydro(s: dict, off, lst, params: OrcParams, want_ngb_acc: bool = False):
    n = s["x"].size
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "du", "vsig")}
    nacc = np.zeros(max(int(off[-1]), 1)) if want_ngb_acc else None
    lib().orc_hydro(n, *[_f64(s[k]) for k in ("x", "y", "z", "range", "vx", "vy", "vz", "m", "rho", "P",
                                               "divv", "curlv", "omega", "psi")],
                    np.ascontiguousarray(off, np.int64), np.ascontiguousarray(lst, np.int32),
                    out["ax"], out["ay"], out["az"], out["du"], out["vsig"],
                    nacc.ctypes.data_as(C.c_void_p) if nacc is not None else None, C.byref(params))
    if want_ngb_acc:
        out["ngb_acc"] = nacc[: int(off[-1])]
    return out


def gravity(x, y, z, m, rng, params: OrcParams, targets=None):
    x, y, z, m, rng = _f64(x), _f64(y), _f64(z), _f64(m), _f64(rng)
    n = x.size
    if targets is None:
        nt, tp = n, None
    else:
        targets = np.ascontiguousarray(targets, np.int32)
        nt, tp = targets.size, targets.ctypes.data_as(C.c_void_p)
    g = [np.zeros(nt) for _ in range(4)]
    lib().orc_gravity(nt, tp, n, x, y, z, m, rng, *g, C.byref(params))
    return g


# ---------------------------------------------------------------------------
# the same loops for a sample of target particles against the whole state
# (parity checks at the full workload sizes)
# ---------------------------------------------------------------------------
def _tgt(targets):
    return np.ascontiguousarray(targets, np.int32)


def solve_range_sample(x, y, z, range0, targets, params: OrcParams):
    """h solve of the targets only (all particles are candidates), each from
    its guess range0[target]: (range, n_ngb, evaluations) per target."""
    x, y, z, r0, t = _f64(x), _f64(y), _f64(z), _f64(range0), _tgt(targets)
    rng = np.zeros(t.size)
    nn = np.zeros(t.size, np.int32)
    ne = np.zeros(t.size, np.int32)
    lib().orc_solve_range_tgt(t.size, t, x.size, x, y, z, r0, rng, nn, ne, C.byref(params))
    return rng, nn, ne


def find_ngb_sample(x, y, z, range_t, targets):
    """Exact lists {j : ds2 < range_t[t]^2} (ascending j) of the targets, as
    CSR over the targets."""
    x, y, z, rt, t = _f64(x), _f64(y), _f64(z), _f64(range_t), _tgt(targets)
    cnt = np.zeros(t.size, np.int32)
    off = np.zeros(t.size + 1, np.int64)
    tot = lib().orc_find_ngb_tgt(t.size, t, x.size, x, y, z, rt, cnt, off, None)
    lst = np.zeros(max(tot, 1), np.int32)
    lib().orc_find_ngb_tgt(t.size, t, x.size, x, y, z, rt, cnt, off, lst.ctypes.data_as(C.c_void_p))
    return cnt, off, lst[:tot]


def density_sample(s: dict, targets, off, lst):
    """Density loop of the targets over their lists (find_ngb_sample's CSR)."""
    t = _tgt(targets)
    out = {k: np.zeros(t.size) for k in ("rho", "divv", "curlv", "omega", "psi")}
    lib().orc_density_tgt(t.size, t, *[_f64(s[k]) for k in ("x", "y", "z", "range", "vx", "vy", "vz", "m")],
                          np.ascontiguousarray(off, np.int64), np.ascontiguousarray(lst, np.int32),
                          out["rho"], out["divv"], out["curlv"], out["omega"], out["psi"])
    return out


def hydro_sample(s: dict, targets, params: OrcParams):
    """Hydro derivatives of the targets, i-side and j-side, over the whole
    state s (per-particle fields of every particle taken as given)."""
    t = _tgt(targets)
    out = {k: np.zeros(t.size) for k in ("ax", "ay", "az", "du", "vsig")}
    lib().orc_hydro_tgt(t.size, t, s["x"].size, *[_f64(s[k]) for k in (
        "x", "y", "z", "range", "vx", "vy", "vz", "m", "rho", "P", "divv", "curlv", "omega", "psi")],
        out["ax"], out["ay"], out["az"], out["du"], out["vsig"], C.byref(params))
    return out


def gravity_sources(x, y, z, m, rng, params: OrcParams, targets, jlo: int, jhi: int):
    """Gravity on `targets` from the sources [jlo, jhi) only."""
    x, y, z, m, rng = _f64(x), _f64(y), _f64(z), _f64(m), _f64(rng)
    targets = np.ascontiguousarray(targets, np.int32)
    g = [np.zeros(targets.size) for _ in range(4)]
    lib().orc_gravity_src(targets.size, targets.ctypes.data_as(C.c_void_p), x.size, int(jlo), int(jhi), x, y, z, m,
                          rng, *g, C.byref(params))
    return g


def morton_keys(x, y, z):
    x, y, z = _f64(x), _f64(y), _f64(z)
    k = np.zeros(x.size, np.uint64)
    box = np.zeros(4)
    lib().orc_morton_keys(x.size, x, y, z, k, box.ctypes.data_as(C.c_void_p))
    return k, box


def peano_keys(x, y, z):
    """Peano-Hilbert keys of positions as CUDAsph::sort_bodies makes them
    (sort_bodies.cpp:121-160, float quantisation, 18 bits per dimension)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    k = np.zeros(x.size, np.uint64)
    box = np.zeros(4)
    lib().orc_peano_keys(x.size, x, y, z, k, box.ctypes.data_as(C.c_void_p))
    return k, box


def peano_hilbert_key(x, y, z, bits):
    """peano_hilbert_key of one integer triplet (sort_bodies.cpp:66-105)."""
    return int(lib().orc_peano_hilbert_key(int(x), int(y), int(z), int(bits)))


def sort_order(keys):
    keys = np.ascontiguousarray(keys, np.uint64)
    o = np.zeros(keys.size, np.int32)
    lib().orc_sort_order(keys.size, keys, o)
    return o


STATE_FIELDS = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "rho", "P", "u", "mu", "divv", "curlv", "omega",
                "psi", "ax", "ay", "az", "du", "gx", "gy", "gz", "phi", "vsig")


class Sim:
    """Whole-step oracle (step.cpp:13-147) over a dict of float64 arrays."""

    def __init__(self, ic: dict, params: OrcParams):
        n = ic["x"].size
        self.n = n
        self.params = params
        self.arr = {}
        for k in STATE_FIELDS:
            self.arr[k] = _f64(ic[k]).copy() if k in ic else np.zeros(n)
        self.n_ngb = np.zeros(n, np.int32)
        self.st = OrcState()
        self.st.n = n
        for k in STATE_FIELDS:
            setattr(self.st, k, self.arr[k].ctypes.data_as(C.POINTER(C.c_double)))
        self.st.n_ngb = self.n_ngb.ctypes.data_as(C.POINTER(C.c_int))
        self.st.dt = float(ic.get("dt", 0.0))
        self.st.time = float(ic.get("time", 0.0))
        self.st.iteration = 0

    def step(self):
        lib().orc_step(C.byref(self.st), C.byref(self.params))

    @property
    def dt(self):
        return self.st.dt

    @property
    def time(self):
        return self.st.time

    def stats(self):
        return np.array(self.st.stats[:14])


# ---------------------------------------------------------------------------
# the reference built for the host (oracle/_ref/libref_cpu.so), FP32
# ---------------------------------------------------------------------------
_f4p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.exists(REF_PATH):
        raise FileNotFoundError(f"{REF_PATH} not built (make -C oracle ref needs the reference tree)")
    L = C.CDLL(REF_PATH)
    L.ref_kernel_eval.argtypes = [C.c_int, C.c_int, _fp, _fp]
    L.ref_pressure.argtypes = [C.c_int, _fp, _fp, _fp, _fp]
    L.ref_find_root.argtypes = [C.c_float, C.c_float]
    L.ref_find_root.restype = C.c_float
    L.ref_peano_key.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.ref_peano_key.restype = C.c_longlong
    L.ref_build_kdtree.argtypes = [C.c_int, _fp, _fp, C.c_void_p]
    L.ref_solve_range.argtypes = [C.c_int, _fp, _ip, _fp, C.c_float]
    L.ref_ngb_offsets.argtypes = [C.c_int, _ip, _ip]
    L.ref_ngb_offsets.restype = C.c_int
    L.ref_find_ngb.argtypes = [C.c_int, _fp, _fp, _ip, _ip, C.c_void_p]
    L.ref_density.argtypes = [C.c_int, _fp, _fp, _ip, _ip, _ip, _fp, _fp]
    L.ref_hydro.argtypes = [C.c_int, _fp, _fp, _fp, _fp, _ip, _ip, _ip, _fp, _fp, _fp, C.c_float, C.c_float]
    L.ref_add_ngb_acc.argtypes = [C.c_int, _fp, _ip, _ip, _ip, _fp, _fp]
    L.ref_gravity.argtypes = [C.c_int, C.c_void_p, C.c_int, _fp, _fp, _fp]
    L.ref_num_threads.restype = C.c_int
    _ref = L
    return L


def _f4(*cols):
    return np.ascontiguousarray(np.stack([np.asarray(c, np.float32) for c in cols], axis=1))


class RefPipeline:
    """One pass of the reference's SPH accelerations (sph_accelerations.cpp:3-121)
    and gravity (CUDA_gravity.cpp:3-71) with the reference's own FP32 code."""

    def __init__(self, s: dict):
        self.n = n = s["x"].size
        self.pos = _f4(s["x"], s["y"], s["z"], s["range"])
        self.vel = _f4(s["vx"], s["vy"], s["vz"], s["m"])
        self.hydro = _f4(np.zeros(n), np.zeros(n), s["u"], s["mu"])

    def kdtree(self):
        n = self.n
        self.nodes = np.zeros((n + 1, 4), np.float32)
        ref().ref_build_kdtree(n, self.pos, self.nodes, None)
        return self.nodes

    def solve_range(self, rel_err=1e-3):
        self.n_ngb = np.zeros(self.n, np.int32)
        ref().ref_solve_range(self.n, self.pos, self.n_ngb, self.nodes, rel_err)
        return self.pos[:, 3].copy(), self.n_ngb.copy()

    def find_ngb(self):
        n = self.n
        self.off = np.zeros(n + 1, np.int32)
        # the reference sizes lists from solve_range's count; one extra slot
        # per particle absorbs the round-off case in which find_ngb's walk
        # (dev_find_ngb.cu:67) admits one more neighbour than that count
        # (dev_solve_range.cu:142)
        tot = ref().ref_ngb_offsets(n, self.n_ngb + 1, self.off)
        self.lst = np.full(tot, -1, np.int32)
        walk = np.zeros(n, np.int32)
        ref().ref_find_ngb(n, self.pos, self.nodes, self.off, self.lst, walk.ctypes.data_as(C.c_void_p))
        # recount from the list (a -1 sentinel ends each written run)
        cnt = np.zeros(n, np.int32)
        for i in range(n):
            seg = self.lst[self.off[i]:self.off[i + 1]]
            k = np.argmax(seg < 0) if (seg < 0).any() else seg.size
            cnt[i] = k
        self.n_ngb = cnt
        return cnt, self.off, self.lst

    def density(self):
        self.ddata = np.zeros((self.n, 4), np.float32)
        ref().ref_density(self.n, self.pos, self.vel, self.n_ngb, self.off, self.lst, self.hydro, self.ddata)
        return self.hydro[:, 0].copy(), self.ddata.copy()

    def pressure(self):
        P = np.zeros(self.n, np.float32)
        ref().ref_pressure(self.n, np.ascontiguousarray(self.hydro[:, 0]), np.ascontiguousarray(self.hydro[:, 2]),
                           np.ascontiguousarray(self.hydro[:, 3]), P)
        self.hydro[:, 1] = P
        return P

    def hydro_dots(self, alpha=1.0, beta=2.0):
        n = self.n
        self.dots = np.zeros((n, 4), np.float32)
        self.vsig = np.zeros(n, np.float32)
        self.ngb_acc = np.zeros(self.lst.size, np.float32)
        ref().ref_hydro(n, self.pos, self.vel, self.hydro, self.ddata, self.n_ngb, self.off, self.lst,
                        self.dots, self.vsig, self.ngb_acc, alpha, beta)
        ref().ref_add_ngb_acc(n, self.pos, self.n_ngb, self.off, self.lst, self.ngb_acc, self.dots)
        return self.dots.copy(), self.vsig.copy()

    def time_step(self, n_grav_targets: int = 256, seed: int = 0) -> dict:
        """Wall-clock of one reference step on this state (sph_accelerations.cpp:
        3-121 + CUDA_gravity.cpp:3-71): kd-tree build (the reference's host
        code, single thread), solve_range / find_ngb / density / pressure /
        hydro / j-side scatter over all particles (OpenMP over particles), and
        gravity for a seeded sample of n_grav_targets bodies against all n,
        extrapolated to n.  Returns the per-phase seconds and 'step'."""
        import time
        t = {}
        t0 = time.perf_counter(); self.kdtree(); t["tree"] = time.perf_counter() - t0
        t0 = time.perf_counter(); self.solve_range(); t["solve_range"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        n = self.n
        self.off = np.zeros(n + 1, np.int32)
        tot = ref().ref_ngb_offsets(n, self.n_ngb + 4, self.off)
        self.lst = np.full(tot, -1, np.int32)
        ref().ref_find_ngb(n, self.pos, self.nodes, self.off, self.lst, None)
        t["find_ngb"] = time.perf_counter() - t0
        t0 = time.perf_counter(); self.density(); t["density"] = time.perf_counter() - t0
        t0 = time.perf_counter(); self.pressure(); t["pressure"] = time.perf_counter() - t0
        t0 = time.perf_counter(); self.hydro_dots(); t["hydro"] = time.perf_counter() - t0
        tg = np.random.default_rng(seed).choice(n, size=min(n_grav_targets, n), replace=False).astype(np.int32)
        t0 = time.perf_counter(); self.gravity(tg); tgs = time.perf_counter() - t0
        t["gravity_sample"] = tgs
        t["gravity"] = tgs * n / tg.size
        t["step"] = sum(v for k, v in t.items() if k != "gravity_sample")
        return t

    def gravity(self, targets=None):
        n = self.n
        gpos = _f4(self.pos[:, 0], self.pos[:, 1], self.pos[:, 2], self.vel[:, 3])
        gvel = _f4(self.vel[:, 0], self.vel[:, 1], self.vel[:, 2], self.pos[:, 3].astype(np.float32) ** 2)
        if targets is None:
            nt, tp = n, None
        else:
            targets = np.ascontiguousarray(targets, np.int32)
            nt, tp = targets.size, targets.ctypes.data_as(C.c_void_p)
        out = np.zeros((nt, 4), np.float32)
        ref().ref_gravity(nt, tp, n, gpos, gvel, out)
        return out
