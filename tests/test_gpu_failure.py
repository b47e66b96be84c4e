"""Failure reporting without faulting the GPU: host-made bad inputs and
undersized capacities must come back as status flags / error codes, and the
context must stay usable (the reference exits the process instead,
host_calls.cu:14-22, sph_accelerations.cpp:66-72)."""
import numpy as np
import pytest

from cudasph_b200 import ics
from cudasph_b200._capi import FLAG_H_NOT_CONVERGED, FLAG_NGB_OVERFLOW, FLAG_NONFINITE, SphError

pytestmark = pytest.mark.gpu


def _sim(ic, **kw):
    from cudasph_b200.simulation import Simulation, make_params
    base = dict(n_target=32.0, eos_mode=0, soft_mode=1, eps=0.01)
    base.update(kw)
    return Simulation(ic, make_params(**base))


def test_undersized_neighbour_lists_raise_overflow_and_recover():
    ic = ics.polytrope(4096, n_ngb=32, seed=2)
    sim = _sim(ic, ngb_cap=8)
    sim.step()
    assert sim.device_status() & FLAG_NGB_OVERFLOW
    assert np.all(sim.n_ngb() > 8)  # counts are the true counts, the lists truncated
    # the same context continues after the capacity is raised
    from cudasph_b200.simulation import make_params
    sim.set_params(make_params(n_target=32.0, eos_mode=0, soft_mode=1, eps=0.01, ngb_cap=0))
    sim.step()
    assert sim.device_status() & FLAG_NGB_OVERFLOW == 0
    assert np.all(np.isfinite(sim.get("ax")))
    sim.close()


def test_nonfinite_thermal_energy_is_flagged():
    ic = ics.polytrope(2048, n_ngb=32, seed=3)
    ic["u"] = ic["u"].copy()
    ic["u"][100] = np.nan
    sim = _sim(ic)
    sim.step()
    assert sim.device_status() & FLAG_NONFINITE
    sim.close()


def test_h_solve_iteration_limit_is_flagged():
    ic = ics.polytrope(2048, n_ngb=32, seed=4)
    ic["range"] = ic["range"] * 1.7  # far from the root
    sim = _sim(ic, max_iter=1)
    sim.step()
    assert sim.device_status() & FLAG_H_NOT_CONVERGED
    sim.close()


def test_phase_out_of_order_is_an_error_not_a_fault():
    ic = ics.polytrope(1024, n_ngb=32, seed=5)
    sim = _sim(ic)
    with pytest.raises(SphError, match="status 5"):
        sim.density()  # no neighbour lists yet
    with pytest.raises(SphError, match="status 5"):
        sim.adjoint()  # no step kept
    sim.step()
    assert np.all(np.isfinite(sim.get("x")))
    sim.close()
