"""ctypes binding of libcudasph_b200.so (the C ABI in include/cudasph_b200.h).

The library is built in-tree (``python -m cudasph_b200.build``).  There is no
fallback: if the shared library is missing or fails to load, importing the
binding raises, so nothing can silently run on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcudasph_b200.so")

FIELDS = ("x", "y", "z", "range", "vx", "vy", "vz", "m", "rho", "P", "u", "mu", "divv", "curlv", "omega", "psi",
          "ax", "ay", "az", "du", "gx", "gy", "gz", "phi", "vsig")
FIELD_ID = {k: i for i, k in enumerate(FIELDS)}

STATS = ("W", "T", "U", "E", "Jx", "Jy", "Jz", "Rcm_x", "Rcm_y", "Rcm_z", "Vcm_x", "Vcm_y", "Vcm_z", "Mtot",
         "Fx", "Fy", "Fz", "Tx", "Ty", "Tz", "ngb_mean", "ngb_sigma", "ngb_min", "ngb_max", "dt_vel", "dt_eth",
         "dt", "time", "dt_old")
PHASES = ("sort", "predict", "tree", "solve_range", "find_ngb", "density", "pressure", "hydro", "gravity", "finish",
          "kick", "adjoint")

ADJ_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "u", "ax", "ay", "az", "du", "rho")
ADJ_ID = {k: i for i, k in enumerate(ADJ_FIELDS)}

FLAG_NGB_OVERFLOW = 0x1
FLAG_STACK_OVERFLOW = 0x2
FLAG_NONFINITE = 0x4
FLAG_H_NOT_CONVERGED = 0x8

EOS = {"ideal": 0, "gas_radiation": 1}
SOFT = {"spline": 0, "plummer": 1}
PREC = {"fp64": 0, "mixed": 1}


class Params(C.Structure):
    _fields_ = [
        ("n_target", C.c_double), ("rel_err", C.c_double), ("max_iter", C.c_int), ("f_scale", C.c_double),
        ("av_alpha", C.c_double), ("av_beta", C.c_double), ("gamma", C.c_double), ("eos_mode", C.c_int),
        ("soft_mode", C.c_int), ("eps", C.c_double), ("use_psi", C.c_int), ("cn1", C.c_double),
        ("cn2", C.c_double), ("G", C.c_double), ("precision", C.c_int), ("ngb_cap", C.c_int),
        ("sort_every", C.c_int), ("mixed_sph", C.c_int), ("grav_mode", C.c_int), ("theta", C.c_double),
        ("key_mode", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cudasph_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    L.cudasph_default_params.restype = Params
    L.cudasph_create.argtypes = [C.POINTER(Params), ip, ip, C.POINTER(vp)]
    L.cudasph_destroy.argtypes = [vp]
    L.cudasph_last_error.restype = C.c_char_p
    L.cudasph_set_params.argtypes = [vp, C.POINTER(Params)]
    L.cudasph_get_params.argtypes = [vp, C.POINTER(Params)]
    L.cudasph_set_field.argtypes = [vp, ip, vp, ip]
    L.cudasph_get_field.argtypes = [vp, ip, vp, ip]
    L.cudasph_set_state.argtypes = [vp, vp, ip]
    L.cudasph_get_state.argtypes = [vp, vp, ip]
    L.cudasph_get_n_ngb.argtypes = [vp, vp, ip]
    L.cudasph_get_order.argtypes = [vp, vp]
    L.cudasph_set_time.argtypes = [vp, dp, dp]
    L.cudasph_get_time.argtypes = [vp, C.POINTER(dp), C.POINTER(dp)]
    L.cudasph_get_neighbours.argtypes = [vp, vp, vp, vp]
    L.cudasph_get_solve_evals.argtypes = [vp, vp]
    for name in ("begin_step", "shard_pack", "shard_unpack", "sort", "predict", "build_tree", "solve_range", "find_ngb", "density", "pressure", "hydro",
                 "sph_accelerations", "gravity", "finish", "kick", "step", "synchronize", "reset_counters"):
        getattr(L, "cudasph_" + name).argtypes = [vp]
    L.cudasph_steps.argtypes = [vp, ip]
    L.cudasph_step_host.argtypes = [vp, vp, vp]
    L.cudasph_statistics.argtypes = [vp, vp]
    L.cudasph_device_status.argtypes = [vp, C.POINTER(C.c_uint)]
    L.cudasph_set_profiling.argtypes = [vp, ip]
    L.cudasph_phase_times.argtypes = [vp, vp, vp]
    L.cudasph_kernel_launches.argtypes = [vp]
    L.cudasph_kernel_launches.restype = C.c_longlong
    L.cudasph_num_particles.argtypes = [vp]
    L.cudasph_sort_scratch_bytes.argtypes = [ip]
    L.cudasph_sort_scratch_bytes.restype = C.c_size_t
    L.cudasph_morton_keys.argtypes = [ip, vp, vp, vp, vp, vp, vp]
    L.cudasph_peano_keys.argtypes = [ip, vp, vp, vp, vp, vp, vp]
    L.cudasph_peano_hilbert_keys.argtypes = [ip, vp, vp, vp, ip, vp, vp]
    L.cudasph_radix_sort_u64.argtypes = [ip, vp, vp, vp, vp]
    L.cudasph_gravity_direct.argtypes = [ip, vp, vp, vp, ip, dp, dp, ip, vp]
    L.cudasph_fma_peak.argtypes = [ip, ip, vp]
    L.cudasph_fma_peak.restype = C.c_double
    L.cudasph_l2_peak.argtypes = [ip, vp]
    L.cudasph_l2_peak.restype = C.c_double
    L.cudasph_set_keep.argtypes = [vp, ip]
    L.cudasph_set_graph.argtypes = [vp, ip]
    L.cudasph_adjoint_set_field.argtypes = [vp, ip, vp, ip]
    L.cudasph_adjoint_get_field.argtypes = [vp, ip, vp, ip]
    L.cudasph_adjoint_set_dt.argtypes = [vp, dp]
    L.cudasph_adjoint_get_dt.argtypes = [vp, C.POINTER(dp)]
    L.cudasph_adjoint.argtypes = [vp]
    L.cudasph_shard_range.argtypes = [C.c_longlong, ip, ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.cudasph_set_shard.argtypes = [vp, ip, ip]
    L.cudasph_get_shard.argtypes = [vp, vp, vp, vp, vp]
    L.cudasph_device_buffer.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(C.c_longlong)]
    L.cudasph_get_stream.argtypes = [vp, C.POINTER(vp)]
    _lib = L
    return L


class SphError(RuntimeError):
    pass


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = lib().cudasph_last_error().decode(errors="replace")
        raise SphError(f"{what} failed with status {rc}: {msg}")


# names of the symbols the C header declares (for the export test)
def declared_symbols(header_paths):
    import re
    names = []
    for p in header_paths:
        txt = open(p).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.append(name)
    return sorted(set(names))
