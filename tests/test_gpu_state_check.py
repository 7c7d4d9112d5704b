"""Device state check (rh_check_state, rh_set_state_check,
rh_batch_set_state_check): the reference's debug scan of uold after set_uold
(check_nan_kernel, gpu/gpu_utils.cuf:90-118) and cmpdt's negative-pressure
stop (hydro/godunov_utils.f90:278-287).  Bad cells are planted in host
states (bad data, not a device fault): a NaN, a negative density and a cell
whose energy is below its kinetic energy."""
import numpy as np
import pytest

from ramses2_b200._abi import HydroParams
from ramses2_b200._lib import RHError
from ramses2_b200.batch import Batch, dense_to_octs, ic_host, ic_split, problem
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import sedov3d, uniform_mesh

pytestmark = pytest.mark.gpu


def plant(u):
    """Three bad cells: oct 6 cell 3 NaN density (bit 1), oct 10 cell 2
    negative density (bit 2), oct 13 cell 1 energy below kinetic (bit 4);
    returns (count, first oct 1-based, mask)."""
    u[5, 0, 3] = np.nan
    u[9, 0, 2] = -1.0
    r, m1 = u[12, 0, 1], 2.0 * np.sqrt(u[12, 0, 1])
    u[12, 1, 1] = m1
    u[12, 4, 1] = 0.25 * m1 * m1 / r  # E < |m|^2 / (2 rho)
    return 3, 6, 7


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
def test_check_state_finds_planted_cells(prec):
    m = uniform_mesh(4, nsubgrid=1, bc="outflow")
    sedov3d(m)
    P = HydroParams.make(gamma=1.4)
    gpu = GodunovGPU(m, P, precision=prec)
    try:
        assert gpu.check_state(4) == (0, 0, 0)
        u = m.uold.copy()
        want = plant(u)
        gpu.push_uold(u)
        assert gpu.check_state(4) == want
    finally:
        gpu.close()


def test_coarse_step_with_state_check():
    """Switched on, rh_coarse_step returns RH_EBADSTATE after a step that
    leaves a bad cell, and changes nothing on a clean run."""
    m = uniform_mesh(4, nsubgrid=1, bc="outflow")
    sedov3d(m)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    u0 = m.uold.copy()
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        gpu.coarse_step()
        gpu.coarse_step()
        plain = gpu.fetch_uold()
        gpu.push_uold(u0)
        gpu.set_state_check(True)
        gpu.coarse_step()
        gpu.coarse_step()
        assert np.array_equal(gpu.fetch_uold(), plain)
        bad = u0.copy()
        plant(bad)
        gpu.push_uold(bad)
        with pytest.raises(RHError, match="RH_EBADSTATE"):
            gpu.coarse_step(1e-3)
    finally:
        gpu.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
def test_batch_state_check_stops_only_the_bad_problem(prec):
    g = 1.4
    good_ic = ic_split(0, [1.0, 0, 0, 0, 1.0], [0.125, 0, 0, 0, 0.1])
    dense = np.empty((5, 16, 16, 16))
    dense[0], dense[1:4], dense[4] = 1.0, 0.0, 2.5
    octs = dense_to_octs(dense)
    octs[17, 0, 4] = np.nan
    results = {}
    for on in (False, True):
        b = Batch(prec, pool_octs=1 << 12)
        try:
            b.set_state_check(on)
            ok = b.add(problem((16, 8, 8), gamma=g, max_steps=4), good_ic)
            if on:
                badid = b.add(problem((16, 16, 16), gamma=g, max_steps=4), ic_host(octs))
            b.step(4)
            done, nstep, _ = b.poll()
            assert done[ok] == 1 and nstep[ok] == 4
            results[on] = b.fetch(ok)
            if on:
                assert done[badid] == 2 and nstep[badid] == 1
                assert b.check_mask(badid) & 1
                assert b.check_mask(ok) == 0
        finally:
            b.close()
    assert np.array_equal(results[False], results[True])


def test_server_reports_a_failed_request():
    from ramses2_b200.serve import HydroServer, Request

    dense = np.empty((5, 16, 16, 16))
    dense[0], dense[1:4], dense[4] = 1.0, 0.0, 2.5
    octs = dense_to_octs(dense)
    octs[3, 0, 0] = -2.0  # negative density
    reqs = [Request(0, 0.0, problem((16, 16, 16), max_steps=6), ic_split(1, [1, 0, 0, 0, 1], [0.2, 0, 0, 0, 0.1])),
            Request(1, 0.0, problem((16, 16, 16), max_steps=6), ic_host(octs)),
            Request(2, 0.0, problem((32, 16, 16), max_steps=6), ic_split(2, [1, 0, 0, 0, 1], [0.3, 0, 0, 0, 0.2]))]
    srv = HydroServer("fp32_bulk", pool_bytes=64 << 20, chunk=2, state_check=True)
    try:
        st = srv.run(reqs, realtime=False)
    finally:
        srv.close()
    assert st["failed"] == 1 and st["served"] == 2
    assert reqs[1].failed and not reqs[0].failed and not reqs[2].failed
    assert reqs[0].nsteps == 6 and reqs[2].nsteps == 6
