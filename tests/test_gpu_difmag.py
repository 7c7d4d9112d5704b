"""Artificial diffusion (difmag > 0: unsplit's cmpdivu / cmpdiff,
hydro/umuscl.f90:2392-2540) through rh_coarse_step against the FP64 CPU
oracle, and the configurations the library refuses.

Bar: relative L1 <= 1e-12 per conserved variable per step from the same
state and dt, and the next dt (courant_fine of the diffused state) within
1e-12."""
import numpy as np
import pytest

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200._lib import RHError
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import prim_to_cons, sedov_amr_mesh, uniform_mesh

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def rel_l1(a, b):
    num = np.abs(a - b).sum(axis=(0, 2))
    den = np.abs(b).sum(axis=(0, 2))
    return num / np.where(den > 0, den, 1.0)


def compressive_state(mesh, seed, gamma=1.4):
    """A flow converging on the box centre (where the diffusion acts) and
    diverging at the faces, with random density and velocity perturbations
    and a pressure blob."""
    rng = np.random.default_rng(seed)
    lev = mesh.levelmin
    n = 2 * (1 << (lev - 1))
    x = (np.arange(n) + 0.5) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    rho = 1.0 + 0.5 * rng.random((n, n, n))
    u, v, w = (-0.8 * np.sin(2 * np.pi * (c - 0.5)) + 0.1 * rng.standard_normal((n, n, n)) for c in (xx, yy, zz))
    p = 1.0 + 5.0 * np.exp(-((xx - 0.3) ** 2 + (yy - 0.6) ** 2 + (zz - 0.45) ** 2) / 0.01)
    mesh.from_dense(prim_to_cons(rho, u, v, w, p, gamma), lev)
    return gamma


@pytest.mark.parametrize("bc,gravity,riemann", [("outflow", (0.0, 0.0, 0.0), "hllc"),
                                                ("periodic", (0.0, 0.0, 0.0), "llf"),
                                                ("reflexive", (0.3, -0.2, 0.5), "hllc")])
def test_diffusion_steps_match_oracle(bc, gravity, riemann):
    m = uniform_mesh(5, nsubgrid=1, bc=bc, gravity=gravity)
    g = compressive_state(m, 3)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann=riemann, difmag=0.2)
    P0 = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann=riemann)
    u0 = m.uold.copy()
    mo = uniform_mesh(5, nsubgrid=1, bc=bc, gravity=gravity)
    mo.uold[:] = u0
    o = oracle.OracleHydro(mo, P)
    gpu = GodunovGPU(m, P)
    try:
        # the same state and dt every step: the diffused step agrees
        for step in range(3):
            gpu.push_uold(mo.uold)
            dto, _ = o.step_uniform()
            gpu.coarse_step(dto)
            err = rel_l1(gpu.fetch_uold(), mo.uold)
            assert np.all(err <= TOL_FP64), (step, err)
        # the diffusion is not negligible here: the same step without it differs
        plain = uniform_mesh(5, nsubgrid=1, bc=bc, gravity=gravity)
        plain.uold[:] = u0
        dtp, _ = oracle.OracleHydro(plain, P0).step_uniform()
        mo2 = uniform_mesh(5, nsubgrid=1, bc=bc, gravity=gravity)
        mo2.uold[:] = u0
        oracle.OracleHydro(mo2, P).step_uniform(dtp)
        assert np.max(rel_l1(mo2.uold, plain.uold)) > 1e-6
        # the GPU's own trajectory, its dt from the diffused state each step
        gpu.push_uold(u0)
        mo.uold[:] = u0
        for step in range(3):
            dto, _ = o.step_uniform()
            dtg = gpu.coarse_step()
            assert dtg == pytest.approx(dto, rel=1e-12), step
        err = rel_l1(gpu.fetch_uold(), mo.uold)
        assert np.all(err <= 1e-11), err
    finally:
        gpu.close()


def test_host_step_with_diffusion_equals_the_device_step():
    m = uniform_mesh(5, nsubgrid=1, bc="outflow")
    g = compressive_state(m, 9)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", difmag=0.3)
    u0 = m.uold.copy()
    gpu = GodunovGPU(m, P)
    try:
        gpu.push_uold(u0)
        dt = gpu.coarse_step()
        dev = gpu.fetch_uold()
        host = u0.copy()
        dt_h, _ = gpu.coarse_step_host(host)
        assert dt_h == dt
        assert np.array_equal(host, dev)
    finally:
        gpu.close()


def test_diffusion_refused_outside_one_fp64_level():
    m = uniform_mesh(4, nsubgrid=1, bc="outflow")
    g = compressive_state(m, 1)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", difmag=0.1)
    gpu = GodunovGPU(m, P, precision="fp32_bulk")
    try:
        with pytest.raises(RHError, match="difmag"):
            gpu.coarse_step()
    finally:
        gpu.close()
    ma, ga = sedov_amr_mesh(3, 5, radius=0.3)
    assert all(ma.noct[l] for l in (3, 4, 5))
    PA = HydroParams.make(gamma=ga, courant_factor=0.8, slope_type=2, riemann="hllc", difmag=0.1,
                          interpol_var=0, interpol_type=1)
    gpu = GodunovGPU(ma, PA)
    try:
        with pytest.raises(RHError, match="difmag"):
            gpu.coarse_step()
        PA.difmag = 0.0
        gpu.coarse_step()  # the same mesh steps without it
    finally:
        gpu.close()
