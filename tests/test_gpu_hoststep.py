"""rh_coarse_step_host: a coarse step of a host-resident state with the copies
overlapped with the pencils must give, bit for bit, what
rh_set_grid_device + rh_coarse_step + rh_transfer_grid_host give, for both
precisions and for boundaries that wrap (every pencil then needs the last
chunks) and that clamp; its dt_next must be the courant_fine dt the separate
calls report for the new state."""
import numpy as np
import pytest

from ramses2_b200._abi import HydroParams
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import sedov3d, uniform_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_host_step_equals_separate_calls(prec, bc):
    m = uniform_mesh(6, nsubgrid=1, bc=bc)  # 32,768 octs: several chunks
    sedov3d(m, radius_cells=3.0)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    u0 = m.uold.copy()
    gpu = GodunovGPU(m, P, precision=prec)
    try:
        # the separate calls, three steps, dt from courant_fine each time
        gpu.push_uold(u0)
        ref, dts = [], []
        for _ in range(3):
            dts.append(gpu.coarse_step())
            ref.append(gpu.fetch_uold())
        lev = m.levelmin
        nxt_ref = min(m.dx(lev) / P.smallc, gpu.courant_fine(lev)[4])
        # the host step: first call computes dt, later calls take the previous dt_next
        h = u0.copy()
        dt, nxt = gpu.coarse_step_host(h)
        assert dt == dts[0]
        assert np.array_equal(h, ref[0])
        assert nxt == dts[1]
        out = np.empty_like(h)
        dt, nxt = gpu.coarse_step_host(h, out, dt=nxt)  # separate output buffer
        assert dt == dts[1] and np.array_equal(out, ref[1]) and nxt == dts[2]
        dt, nxt = gpu.coarse_step_host(out, dt=nxt)     # in place
        assert dt == dts[2] and np.array_equal(out, ref[2])
        assert nxt == nxt_ref
        # the device state is the new one: a plain step continues from it
        gpu.coarse_step(nxt)
    finally:
        gpu.close()


def test_host_step_on_a_multi_level_mesh_makes_the_separate_calls():
    from ramses2_b200.mesh import sedov_amr_mesh

    m, g = sedov_amr_mesh(3, 5, radius=0.3)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0, interpol_type=1)
    u0 = m.uold.copy()
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        dt_ref = gpu.coarse_step()
        ref = gpu.fetch_uold()
        h = u0.copy()
        dt, nxt = gpu.coarse_step_host(h)
        assert dt == dt_ref and np.array_equal(h, ref) and nxt > 0
    finally:
        gpu.close()
