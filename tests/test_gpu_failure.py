"""Failure path of the device waits, exercised without a fault: a bounded
mbarrier wait on a barrier that nothing arrives on gives up, the host gets
RH_ETIMEDOUT from the device error word, and the context keeps working."""
import numpy as np
import pytest

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200._lib import check, lib
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import sedov3d, uniform_mesh

pytestmark = pytest.mark.gpu

RH_ETIMEDOUT = 5


def test_bounded_wait_times_out_and_context_survives():
    L = lib()
    check(L.rh_init(0), "rh_init")
    assert L.rh_selftest_wait(1000) == RH_ETIMEDOUT
    assert "wait bound" in L.rh_last_error().decode()
    assert L.rh_sync() == 0  # the error word was consumed
    m = uniform_mesh(4, nsubgrid=1, bc="outflow")
    sedov3d(m, radius_cells=1.5)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P)
    o.step_uniform()
    ref = m.uold.copy()
    m.uold[:] = u0
    gpu = GodunovGPU(m, P)
    try:
        gpu.step_uniform()
        assert L.rh_sync() == 0
        out = gpu.fetch_uold()
    finally:
        gpu.close()
    err = np.abs(out - ref).sum(axis=(0, 2)) / np.abs(ref).sum(axis=(0, 2))
    assert np.all(err <= 1e-12), err
