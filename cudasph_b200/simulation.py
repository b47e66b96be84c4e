"""Python handle on the device-resident SPH step (test and benchmark harness).

:class:`Simulation` wraps one ``sph_ctx`` of the C ABI.  Its methods carry the
names of the reference driver's member functions (CUDAsph.h:72-163) --
``step``, ``sph_accelerations``, ``CUDA_solve_range``, ``CUDA_gravity``,
``compute_timestep``, ``system_statistics`` -- and call the corresponding
entry points; state is addressed in the caller's original particle order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import FIELDS, FIELD_ID, PHASES, STATS, check, lib


def make_params(**kw) -> _capi.Params:
    """sph_params with the reference's defaults, overridden by keyword.

    String shorthands: eos='ideal'|'gas_radiation', soft='spline'|'plummer',
    precision='fp64'|'mixed'."""
    p = lib().cudasph_default_params()
    if "eos" in kw:
        kw["eos_mode"] = _capi.EOS[kw.pop("eos")]
    if "soft" in kw:
        kw["soft_mode"] = _capi.SOFT[kw.pop("soft")]
    if isinstance(kw.get("precision"), str):
        kw["precision"] = _capi.PREC[kw["precision"]]
    for k, v in kw.items():
        if v is None:
            continue
        setattr(p, k, v)
    return p


class Simulation:
    def __init__(self, ic: dict, params: _capi.Params, device: int = 0):
        self.n = int(np.asarray(ic["x"]).size)
        self.device = device
        self.params = params
        h = C.c_void_p()
        check(lib().cudasph_create(C.byref(params), self.n, device, C.byref(h)), "cudasph_create")
        self._h = h
        self.set_state(ic)
        check(lib().cudasph_set_time(self._h, float(ic.get("time", 0.0)), float(ic.get("dt", 0.0))), "set_time")

    # -- lifecycle ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cudasph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state --------------------------------------------------------------
    def set(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.n
        check(lib().cudasph_set_field(self._h, FIELD_ID[name], a.ctypes.data, 0), f"set_field({name})")

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.n, np.float64)
        check(lib().cudasph_get_field(self._h, FIELD_ID[name], out.ctypes.data, 0), f"get_field({name})")
        return out

    def set_state(self, ic: dict):
        for k in FIELDS:
            if k in ic:
                self.set(k, ic[k])

    def get_state(self, names=FIELDS) -> dict:
        return {k: self.get(k) for k in names}

    def n_ngb(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        check(lib().cudasph_get_n_ngb(self._h, out.ctypes.data, 0), "get_n_ngb")
        return out

    def order(self) -> np.ndarray:
        """original particle id held by each tree slot"""
        out = np.empty(self.n, np.int32)
        check(lib().cudasph_get_order(self._h, out.ctypes.data), "get_order")
        return out

    def solve_evals(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        check(lib().cudasph_get_solve_evals(self._h, out.ctypes.data), "get_solve_evals")
        return out

    def neighbours(self):
        """(counts, offsets, list) in original ids; each list ascending by tree slot."""
        cnt = np.empty(self.n, np.int32)
        off = np.empty(self.n + 1, np.int64)
        check(lib().cudasph_get_neighbours(self._h, cnt.ctypes.data, off.ctypes.data, None), "get_neighbours")
        lst = np.empty(max(int(off[-1]), 1), np.int32)
        check(lib().cudasph_get_neighbours(self._h, cnt.ctypes.data, off.ctypes.data, lst.ctypes.data),
              "get_neighbours")
        return cnt, off, lst[: int(off[-1])]

    @property
    def time(self) -> float:
        t, d = C.c_double(), C.c_double()
        check(lib().cudasph_get_time(self._h, C.byref(t), C.byref(d)), "get_time")
        return t.value

    @property
    def dt(self) -> float:
        t, d = C.c_double(), C.c_double()
        check(lib().cudasph_get_time(self._h, C.byref(t), C.byref(d)), "get_time")
        return d.value

    def set_params(self, params: _capi.Params):
        check(lib().cudasph_set_params(self._h, C.byref(params)), "set_params")
        self.params = params

    # -- phases (reference names) ------------------------------------------
    def _call(self, name):
        check(getattr(lib(), "cudasph_" + name)(self._h), name)

    def sort_bodies(self):
        self._call("sort")

    def predict(self):
        self._call("predict")

    def build_tree(self):
        self._call("build_tree")

    def CUDA_solve_range(self):
        self._call("solve_range")

    def find_ngb(self):
        self._call("find_ngb")

    def density(self):
        self._call("density")

    def pressure(self):
        self._call("pressure")

    def hydro(self):
        self._call("hydro")

    def sph_accelerations(self):
        self._call("sph_accelerations")

    def CUDA_gravity(self):
        self._call("gravity")

    def finish(self):
        self._call("finish")

    def kick(self):
        self._call("kick")

    def step(self, k: int = 1):
        if k == 1:
            self._call("step")
        else:
            check(lib().cudasph_steps(self._h, k), "steps")

    @staticmethod
    def _field_ptrs(fields: dict):
        """pointer array of cudasph_set_state / get_state (float64 C-contiguous arrays)"""
        p = (C.c_void_p * len(FIELDS))()
        for k, i in FIELD_ID.items():
            if k in fields:
                a = fields[k]
                if a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError(f"field {k}: a C-contiguous float64 array is required")
                p[i] = a.ctypes.data
        return p

    def step_host(self, fields_in: dict, fields_out: dict):
        """One step through host buffers (set_state + step + get_state)."""
        check(lib().cudasph_step_host(self._h, self._field_ptrs(fields_in), self._field_ptrs(fields_out)),
              "step_host")

    def set_state_host(self, fields: dict):
        """All given fields from host (or pinned) buffers in one call (one synchronisation)."""
        check(lib().cudasph_set_state(self._h, self._field_ptrs(fields), 0), "set_state")

    def get_state_host(self, fields: dict):
        """All given fields into caller-owned host buffers in one call (one synchronisation)."""
        check(lib().cudasph_get_state(self._h, self._field_ptrs(fields), 0), "get_state")

    def synchronize(self):
        self._call("synchronize")

    def torch_stream(self):
        """The context's CUDA stream as a torch stream (events and collectives
        ordered with the context's work are recorded on it)."""
        if getattr(self, "_stream", None) is None:
            import torch
            s = C.c_void_p()
            check(lib().cudasph_get_stream(self._h, C.byref(s)), "get_stream")
            self._stream = torch.cuda.ExternalStream(s.value or 0, device=f"cuda:{self.device}")
        return self._stream

    def system_statistics(self) -> dict:
        out = np.empty(len(STATS), np.float64)
        check(lib().cudasph_statistics(self._h, out.ctypes.data), "statistics")
        return dict(zip(STATS, out.tolist()))

    def compute_timestep(self) -> float:
        return self.system_statistics()["dt"]

    def device_status(self) -> int:
        f = C.c_uint()
        check(lib().cudasph_device_status(self._h, C.byref(f)), "device_status")
        return f.value

    def set_graph(self, on: bool = True):
        """Replay steady steps from a captured CUDA graph."""
        check(lib().cudasph_set_graph(self._h, int(on)), "set_graph")

    def set_time(self, time: float, dt: float):
        check(lib().cudasph_set_time(self._h, float(time), float(dt)), "set_time")

    # -- discrete adjoint ---------------------------------------------------
    def set_keep(self, on: bool = True):
        """Make every step keep what its reverse sweep (adjoint) needs."""
        check(lib().cudasph_set_keep(self._h, int(on)), "set_keep")

    def adjoint_set(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        check(lib().cudasph_adjoint_set_field(self._h, _capi.ADJ_ID[name], a.ctypes.data, 0), f"adjoint_set({name})")

    def adjoint_get(self, name: str) -> np.ndarray:
        out = np.empty(self.n, np.float64)
        check(lib().cudasph_adjoint_get_field(self._h, _capi.ADJ_ID[name], out.ctypes.data, 0),
              f"adjoint_get({name})")
        return out

    def adjoint_set_dt(self, dtbar: float):
        check(lib().cudasph_adjoint_set_dt(self._h, float(dtbar)), "adjoint_set_dt")

    def adjoint_get_dt(self) -> float:
        d = C.c_double()
        check(lib().cudasph_adjoint_get_dt(self._h, C.byref(d)), "adjoint_get_dt")
        return d.value

    def adjoint(self):
        """Reverse sweep of the last step (taken with set_keep(True))."""
        self._call("adjoint")

    # -- instrumentation ---------------------------------------------------
    def set_profiling(self, on: bool):
        check(lib().cudasph_set_profiling(self._h, int(on)), "set_profiling")

    def phase_times(self) -> dict:
        ms = np.zeros(len(PHASES), np.float64)
        cnt = np.zeros(len(PHASES), np.int32)
        check(lib().cudasph_phase_times(self._h, ms.ctypes.data, cnt.ctypes.data), "phase_times")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(PHASES)}

    def reset_counters(self):
        self._call("reset_counters")

    def kernel_launches(self) -> int:
        return int(lib().cudasph_kernel_launches(self._h))
