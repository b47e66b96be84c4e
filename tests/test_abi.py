"""The C ABI library: loads, exports every symbol the headers declare, carries
the reference's constants as defaults, and validates arguments on the host.
These tests make no compute call and run without a GPU."""
import ctypes as C
import os
import subprocess

import pytest

from cudasph_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("cudasph_b200.h", "cudasph_b200_legacy.h")]

# the reference's extern "C" symbols (CUDAsph.h:22-48, radixsort.cuh:59-61)
REFERENCE_SYMBOLS = [
    "initCUDA", "allocateCUDAarray", "deleteCUDAarray", "copyArrayToDevice", "copyArrayFromDevice",
    "compute_CUDA_gravity", "allocateNBodyArrays", "deleteNBodyArrays", "zallocateNBodyArrays",
    "zdeleteNBodyArrays", "zcopyArrayFromDevice", "zcopyArrayToDevice", "host_solve_range",
    "host_sph_accelerations", "get_device_count", "cuda_set_device", "cuda_set_device0", "cuda_get_device",
    "RadixSort",
]


def _exports():
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def test_library_loads():
    _capi.lib()


def test_every_declared_symbol_is_exported():
    declared = _capi.declared_symbols(HEADERS)
    assert len(declared) > 40
    ex = _exports()
    missing = [s for s in declared if s not in ex]
    assert not missing, missing


def test_reference_boundary_is_exported():
    ex = _exports()
    assert all(s in ex for s in REFERENCE_SYMBOLS)
    assert set(REFERENCE_SYMBOLS) <= set(_capi.declared_symbols(HEADERS))


def test_reference_driver_objects_resolve_against_this_library():
    """Every symbol of the reference's boundary that the reference driver's
    objects import is exported here (the objects are built from the reference
    sources by `make -C oracle driver`, where the reference tree exists)."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    objs = [os.path.join(ref_dir, f) for f in sorted(os.listdir(ref_dir))] if os.path.isdir(ref_dir) else []
    objs = [o for o in objs if os.path.basename(o).startswith("drv_") and o.endswith(".o")]
    if not objs:
        pytest.skip("reference driver objects not built")
    und = set()
    for o in objs:
        out = subprocess.run(["nm", "-u", o], capture_output=True, text=True, check=True).stdout
        und |= {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    wanted = und & set(REFERENCE_SYMBOLS)
    assert {"host_solve_range", "host_sph_accelerations", "compute_CUDA_gravity"} <= wanted
    assert wanted <= _exports()


def test_default_params_are_the_reference_constants():
    p = _capi.lib().cudasph_default_params()
    assert p.n_target == 24.0        # DESIRED_NGB, dev_solve_range.cu:14
    assert p.rel_err == 1e-3         # CUDA_calls.cpp:4
    assert p.max_iter == 20          # MAX_ITER, dev_solve_range.cu:15
    assert p.f_scale == 0.1          # dev_solve_range.cu:92
    assert (p.av_alpha, p.av_beta) == (1.0, 2.0)  # CUDA_calls.cpp:13-14
    assert abs(p.gamma - 5.0 / 3.0) < 1e-15
    assert (p.cn1, p.cn2) == (0.3, 0.2)  # compute_timestep.cpp:4-5
    assert p.eos_mode == 1 and p.soft_mode == 0 and p.precision == 0


@pytest.mark.parametrize("field,value", [("n_target", 0.0), ("rel_err", -1.0), ("eos_mode", 7), ("soft_mode", 3),
                                         ("precision", 5), ("gamma", 1.0), ("ngb_cap", -1)])
def test_invalid_params_rejected_before_any_device_call(field, value):
    L = _capi.lib()
    p = L.cudasph_default_params()
    setattr(p, field, value)
    h = C.c_void_p()
    assert L.cudasph_create(C.byref(p), 100, 0, C.byref(h)) == 2  # SPH_ERR_ARG
    assert not h.value


def test_plummer_needs_positive_eps():
    L = _capi.lib()
    p = L.cudasph_default_params()
    p.soft_mode = 1
    p.eps = 0.0
    h = C.c_void_p()
    assert L.cudasph_create(C.byref(p), 10, 0, C.byref(h)) == 2


def test_null_context_calls_return_arg_error():
    L = _capi.lib()
    for name in ("sort", "predict", "build_tree", "solve_range", "find_ngb", "density", "hydro", "gravity",
                 "finish", "kick", "step"):
        assert getattr(L, "cudasph_" + name)(None) == 2, name
    assert L.cudasph_destroy(None) == 0


def test_create_without_gpu_reports_cuda_error():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    L = _capi.lib()
    p = L.cudasph_default_params()
    h = C.c_void_p()
    assert L.cudasph_create(C.byref(p), 100, 0, C.byref(h)) == 1  # SPH_ERR_CUDA
    assert b"failed" in L.cudasph_last_error()


def test_key_entries_validate_arguments_before_any_device_work():
    """The key entry points reject bad sizes, bit counts and null buffers with
    SPH_ERR_ARG, and return SPH_OK for n = 0, without touching a device."""
    L = _capi.lib()
    for bits in (0, 22, -1):
        assert L.cudasph_peano_hilbert_keys(4, None, None, None, bits, None, None) == 2, bits
    assert L.cudasph_peano_hilbert_keys(-1, None, None, None, 18, None, None) == 2
    assert L.cudasph_peano_hilbert_keys(0, None, None, None, 18, None, None) == 0
    assert L.cudasph_peano_hilbert_keys(4, None, None, None, 18, None, None) == 2
    assert L.cudasph_peano_keys(-1, None, None, None, None, None, None) == 2
    assert L.cudasph_peano_keys(0, None, None, None, None, None, None) == 0
    assert L.cudasph_peano_keys(4, None, None, None, None, None, None) == 2
    assert L.cudasph_morton_keys(4, None, None, None, None, None, None) == 2


def test_key_mode_is_validated():
    L = _capi.lib()
    p = L.cudasph_default_params()
    assert p.key_mode == 0
    p.key_mode = 2
    h = C.c_void_p()
    assert L.cudasph_create(C.byref(p), 100, 0, C.byref(h)) == 2


def test_noalloc_sort_validates_arguments_before_any_device_work():
    """The allocation-free sort rejects a negative size, a size above its
    fixed scratch and null buffers (with a message), and returns SPH_OK for
    n = 0 and n = 1 without touching the buffers (the sentinel addresses
    given here are never dereferenced), all without a device."""
    L = _capi.lib()
    f = L.cudasph_radix_sort_u64_noalloc
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    assert f(-1, None, None, None) == 2
    assert f(262144 + 1, None, None, None) == 2
    assert b"262144" in L.cudasph_last_error()
    assert f(0, None, None, None) == 0
    assert f(1, 0x10, 0x20, None) == 0
    assert f(2, None, 0x20, None) == 2
    assert b"null" in L.cudasph_last_error()
    assert f(2, 0x10, None, None) == 2


def test_gravity_plan_validates_arguments_without_a_device():
    """cudasph_gravity_plan / cudasph_gravity_item reject bad sizes, ranks,
    precisions, softening modes, items and null outputs with SPH_ERR_ARG,
    and answer valid queries, all without a device."""
    L = _capi.lib()
    L.cudasph_gravity_plan.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    L.cudasph_gravity_item.argtypes = [C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p]
    out = (C.c_longlong * 8)()
    assert L.cudasph_gravity_plan(-1, 1, 1, 0, 1, out) == 2
    assert L.cudasph_gravity_plan(4096, 1, 1, 2, 2, out) == 2  # rank >= world
    assert L.cudasph_gravity_plan(4096, 1, 1, 0, 0, out) == 2
    assert L.cudasph_gravity_plan(4096, 7, 1, 0, 1, out) == 2  # precision
    assert L.cudasph_gravity_plan(4096, 1, 5, 0, 1, out) == 2  # softening
    assert L.cudasph_gravity_plan(4096, 1, 1, 0, 1, None) == 2
    assert L.cudasph_gravity_plan(4096, 1, 1, 0, 1, out) == 0
    tile, block, b0, b1, i0, i1, nt, chunk = list(out)
    assert tile == 1024 and nt == 4 and b0 == 0 and b1 * block >= 4096 and i0 == 0 and i1 > 0
    r, a, b = C.c_int(), C.c_int(), C.c_int()
    assert L.cudasph_gravity_item(4096, -1, C.byref(r), C.byref(a), C.byref(b)) == 2
    assert L.cudasph_gravity_item(4096, i1, C.byref(r), C.byref(a), C.byref(b)) == 2
    assert L.cudasph_gravity_item(4096, 0, None, C.byref(a), C.byref(b)) == 2
    assert L.cudasph_gravity_item(4096, 0, C.byref(r), C.byref(a), C.byref(b)) == 0
    assert r.value == 0 and a.value == 1 and b.value > a.value
