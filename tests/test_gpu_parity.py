"""Parity of the CUDA path (through the C ABI) with the FP64 CPU oracle.

Bar (plain FP64 path): relative L1 error <= 1e-12 per conserved variable per
step, on the same input state.  FP32-bulk path: density relative L1 <= 1e-5
against the FP64 oracle.
"""
import os

import numpy as np
import pytest

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200.hydro import GodunovGPU, amr_coarse_step
from ramses2_b200.mesh import riemann3d_state, sedov3d, turbulence3d, uniform_mesh

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32_RHO = 1e-5
NTHREADS = os.cpu_count() or 1


def rel_l1(a, b):
    """Per-variable relative L1 of a vs b, both (N, 5, 8)."""
    num = np.abs(a - b).sum(axis=(0, 2))
    den = np.abs(b).sum(axis=(0, 2))
    return num / np.where(den > 0, den, 1.0)


def blast_state(mesh, seed, gamma):
    """Random 3D Riemann problem + a pressure blob, so every wave family and
    every direction is exercised."""
    rng = np.random.default_rng(seed)
    lev = mesh.levelmin
    n = 2 * (1 << (lev - 1))
    g, dense = riemann3d_state(rng, n, gamma=gamma)
    x = (np.arange(n) + 0.5) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    blob = np.exp(-((xx - 0.3) ** 2 + (yy - 0.6) ** 2 + (zz - 0.45) ** 2) / 0.01)
    dense[4] += 5.0 * blob * dense[4].mean()
    mesh.from_dense(dense, lev)
    return g


def run_one_step(mesh, P, precision="fp64", tile=None, dt=None):
    u0 = mesh.uold.copy()
    o = oracle.OracleHydro(mesh, P, nthreads=NTHREADS)
    dto, cfl_o = o.step_uniform(dt)
    ref = mesh.uold.copy()
    mesh.uold[:] = u0
    gpu = GodunovGPU(mesh, P, precision=precision, tile=tile)
    try:
        dtg, cfl_g = gpu.step_uniform(dt)
        out = gpu.fetch_uold()
    finally:
        gpu.close()
    mesh.uold[:] = u0
    return ref, out, (dto, cfl_o), (dtg, cfl_g)


@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc"])
@pytest.mark.parametrize("slope", [0, 1, 2])
def test_one_step_fp64_solvers_slopes(riemann, slope):
    m = uniform_mesh(5, nsubgrid=2, bc="outflow")
    g = blast_state(m, 11 + slope, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=slope, riemann=riemann)
    ref, out, (dto, co), (dtg, cg) = run_one_step(m, P)
    assert dto == pytest.approx(dtg, rel=1e-13)
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err


@pytest.mark.parametrize("bc,tile", [("outflow", (8, 8, 16)), ("periodic", (7, 7, 3)), ("reflexive", (8, 4, 2))])
@pytest.mark.parametrize("riemann", ["llf", "hllc"])
def test_slope_type3_fp64_and_fp32(bc, tile, riemann):
    """slope_type 3, the positivity-preserving 27-point limiter
    (umuscl.f90:2207-2269): FP64 <= 1e-12 per variable, FP32-bulk density
    <= 1e-5 against the oracle."""
    m = uniform_mesh(5, nsubgrid=1, bc=bc)
    g = blast_state(m, 17, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=3, riemann=riemann)
    ref, out, (dto, _), (dtg, _) = run_one_step(m, P, tile=tile)
    assert dtg == pytest.approx(dto, rel=1e-13)
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err
    ref, out, _, _ = run_one_step(m, P, precision="fp32_bulk", tile=tile)
    err = rel_l1(out, ref)
    assert err[0] <= TOL_FP32_RHO, err


@pytest.mark.parametrize("bc", ["outflow", "periodic", "reflexive",
                                ["periodic", "periodic", "outflow", "outflow", "reflexive", "reflexive"]])
@pytest.mark.parametrize("tile", [(7, 7, 3), (8, 4, 2), (8, 8, 16)])
def test_one_step_fp64_boundaries_tiles(bc, tile):
    m = uniform_mesh(5, nsubgrid=1, bc=bc)
    g = blast_state(m, 3, 1.6)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    ref, out, _, _ = run_one_step(m, P, tile=tile)
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err


def test_courant_fine_parity():
    """Totals agree with an exactly rounded sum (math.fsum) of the cell terms;
    the oracle sums serially (courant_fine.f90:317-386), the GPU by a tree, so
    both are compared with the exact sum rather than with each other."""
    import math

    m = uniform_mesh(5, nsubgrid=2, bc="outflow")
    g = blast_state(m, 5, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    o = oracle.OracleHydro(m, P).courant_fine(5)
    gpu = GodunovGPU(m, P)
    try:
        c = gpu.courant_fine(5)
    finally:
        gpu.close()
    vol = m.dx(5) ** 3
    u = m.uold[m.level_slice(5)]
    mass = math.fsum((u[:, 0, :] * vol).ravel())
    etot = math.fsum((u[:, 4, :] * vol).ravel())
    assert c[0] == pytest.approx(mass, rel=1e-13)
    assert c[1] == pytest.approx(etot, rel=1e-13)
    assert o[0] == pytest.approx(mass, rel=1e-11)
    assert c[2] == pytest.approx(o[2], rel=1e-10)
    assert c[4] == pytest.approx(o[4], rel=1e-13)


def test_sedov_multistep_fp64():
    """Sedov (moncen, HLLC, C=0.8, outflow) at 32^3: both paths
    evolve independently for 12 steps; every step stays within the bar and
    the fused CFL values match the oracle's courant_fine."""
    m = uniform_mesh(5, nsubgrid=1, bc="outflow")
    sedov3d(m)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    mo = uniform_mesh(5, nsubgrid=1, bc="outflow")
    mo.uold[:] = m.uold
    o = oracle.OracleHydro(mo, P, nthreads=NTHREADS)
    gpu = GodunovGPU(m, P)
    try:
        for step in range(12):
            dto, co = o.step_uniform()
            dtg, cg = gpu.step_uniform()
            assert dtg == pytest.approx(dto, rel=1e-12)
            assert cg[0] == pytest.approx(co[0], rel=1e-12)
            err = rel_l1(gpu.fetch_uold(), mo.uold)
            assert np.all(err <= TOL_FP64), (step, err)
    finally:
        gpu.close()


def test_sedov64_per_step_over_100_steps():
    """Sedov 64^3 (levelmin = levelmax = 6, outflow,
    gamma 1.4, E = 1 within 2 cells, moncen, HLLC, C = 0.8), 100 steps.  Each
    step the GPU starts from the oracle's state (rh_set_grid_device) and takes
    the oracle's dt: relative L1 <= 1e-12 per variable at every step.  The
    GPU's own 100-step trajectory ends within 1e-9 of the oracle's."""
    m = uniform_mesh(6, nsubgrid=1, bc="outflow")
    sedov3d(m)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    u0 = m.uold.copy()
    mo = uniform_mesh(6, nsubgrid=1, bc="outflow")
    mo.uold[:] = u0
    o = oracle.OracleHydro(mo, P, nthreads=NTHREADS)
    gpu = GodunovGPU(m, P)
    worst = np.zeros(5)
    try:
        for step in range(100):
            gpu.push_uold(mo.uold)
            dto, _ = o.step_uniform()
            gpu.step_uniform(dto)
            err = rel_l1(gpu.fetch_uold(), mo.uold)
            worst = np.maximum(worst, err)
            assert np.all(err <= TOL_FP64), (step, err)
        final_oracle = mo.uold.copy()
        gpu.push_uold(u0)
        for _ in range(100):
            gpu.step_uniform()
        err = rel_l1(gpu.fetch_uold(), final_oracle)
        assert np.all(err <= 1e-9), err
    finally:
        gpu.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_constant_gravity_one_step(precision):
    """Constant gravity: the half-step velocity predictor of ctoprim
    (umuscl.f90:1739-1901) and the gravity term of cmpdt
    (godunov_utils.f90:228-333) against the oracle."""
    m = uniform_mesh(5, nsubgrid=1, bc="outflow", gravity=(0.3, -0.2, 0.5))
    g = blast_state(m, 5, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    ref, out, (dto, co), (dtg, cg) = run_one_step(m, P, precision=precision)
    err = rel_l1(out, ref)
    if precision == "fp64":
        assert dtg == pytest.approx(dto, rel=1e-13)
        assert np.all(err <= TOL_FP64), err
    else:
        assert dtg == pytest.approx(dto, rel=1e-6)
        assert err[0] <= TOL_FP32_RHO, err


def test_turbulence_one_step_fp64():
    m = uniform_mesh(5, nsubgrid=1, bc="periodic")
    turbulence3d(m, gamma=1.001, mach=5.0)
    P = HydroParams.make(gamma=1.001, courant_factor=0.8, slope_type=1, riemann="hllc")
    ref, out, _, _ = run_one_step(m, P)
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err


@pytest.mark.parametrize("case", ["sedov", "turb", "blast"])
def test_one_step_fp32_bulk(case):
    m = uniform_mesh(5, nsubgrid=1, bc="periodic" if case == "turb" else "outflow")
    gamma = 1.4
    slope = 2
    if case == "sedov":
        sedov3d(m)
    elif case == "turb":
        gamma = 1.001
        slope = 1
        turbulence3d(m, gamma=gamma, mach=5.0)
    else:
        gamma = blast_state(m, 9, 1.4)
    P = HydroParams.make(gamma=gamma, courant_factor=0.8, slope_type=slope, riemann="hllc")
    ref, out, (dto, _), (dtg, _) = run_one_step(m, P, precision="fp32_bulk")
    assert dtg == pytest.approx(dto, rel=1e-6)
    err = rel_l1(out, ref)
    assert err[0] <= TOL_FP32_RHO, err
    assert np.all(err <= 1e-4), err


def test_fp32_bulk_courant_fine_on_its_state():
    """courant_fine of an FP32-bulk state: the values fused into the Godunov
    kernel (FP64 sums and dt over the new FP32 density and momenta and FP64
    energy) and the standalone reduction of the same state re-uploaded both
    match exact sums of the cell terms and the oracle's courant_fine on that
    state (the fetched values are exact: FP32 widened, FP64 energy).  Both
    take the cells in the same FP32-bulk form, so their dt is the same
    number."""
    import math

    m = uniform_mesh(5, nsubgrid=1, bc="outflow")
    g = blast_state(m, 11, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    gpu = GodunovGPU(m, P, precision="fp32_bulk")
    try:
        gpu.step_uniform()
        fused = gpu.courant_fine(5)
        u = gpu.fetch_uold()
        gpu.push_uold(u)
        alone = gpu.courant_fine(5)
    finally:
        gpu.close()
    mo = uniform_mesh(5, nsubgrid=1, bc="outflow")
    mo.uold[:] = u
    o = oracle.OracleHydro(mo, P).courant_fine(5)
    vol = m.dx(5) ** 3
    lu = u[m.level_slice(5)]
    mass = math.fsum((lu[:, 0, :] * vol).ravel())
    etot = math.fsum((lu[:, 4, :] * vol).ravel())
    assert fused[4] == alone[4]
    for c in (fused, alone):
        assert c[0] == pytest.approx(mass, rel=1e-13)
        assert c[1] == pytest.approx(etot, rel=1e-13)
        assert c[2] == pytest.approx(o[2], rel=1e-10)
        assert c[4] == pytest.approx(o[4], rel=1e-13)


# ---------------------------------------------------------------------------
# Coarse-fine (AMR) levels
# ---------------------------------------------------------------------------
def amr_case(bc="outflow", itype=1, ivar=0):
    from ramses2_b200.mesh import amr_mesh, fill_amr_prim

    m = amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.52) ** 2).sum(-1)) < 0.16, bc=bc)

    def prim(x, l):
        r = np.sqrt(((x - 0.5) ** 2).sum(-1))
        rho = 1 + 0.5 * np.exp(-r ** 2 / 0.01)
        p = 1 + 4 * np.exp(-r ** 2 / 0.004)
        z = np.zeros_like(r)
        return rho, 0.3 + z + 0.2 * np.sin(6 * x[..., 1]), -0.2 + z, 0.1 + z * 0 + 0.1 * x[..., 0], p

    fill_amr_prim(m, prim, 1.4)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_type=itype,
                         interpol_var=ivar)
    return m, P


def amr_step(solver, m, dt=None):
    return amr_coarse_step(solver, m, dt)


@pytest.mark.parametrize("bc,itype,ivar,slope", [("outflow", 1, 0, 2), ("periodic", 2, 1, 2), ("reflexive", 0, 0, 2),
                                                 ("outflow", 3, 0, 2), ("outflow", 1, 0, 3)])
def test_amr_steps_fp64(bc, itype, ivar, slope):
    m, P = amr_case(bc, itype, ivar)
    P.slope_type = slope
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    dts = []
    refs = []
    for _ in range(3):
        dts.append(amr_step(o, m))
        refs.append(m.uold.copy())
    m.uold[:] = u0
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        for s in range(3):
            dt = amr_step(gpu, m)
            assert dt == pytest.approx(dts[s], rel=1e-12)
            err = rel_l1(gpu.fetch_uold(), refs[s])
            assert np.all(err <= TOL_FP64), (s, err)
    finally:
        gpu.close()


@pytest.mark.parametrize("bc,itype,ivar,spare", [("outflow", 1, 0, 0), ("periodic", 2, 1, 0), ("outflow", 1, 0, 40)])
def test_amr_coarse_step_native(bc, itype, ivar, spare):
    """rh_coarse_step (the whole level loop in one library call) against the
    oracle's coarse steps, FP64, three steps: same dt, 1e-12 per variable.
    With spare octs beyond the levels (ngridmax larger than the mesh) it
    takes the level-by-level set_unew / set_uold path instead of the levels
    stepped at once and the buffer swap."""
    m, P = amr_case(bc, itype, ivar)
    if spare:
        from ramses2_b200.mesh import Mesh
        big = Mesh(m.grid, m.levelmin, m.levelmax, bc=bc, ngridmax=len(m.grid) + spare)
        big.uold[:len(m.grid)] = m.uold
        big.uold[len(m.grid):] = 7.0  # never part of a level: must come back unchanged
        m = big
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    dts, refs = [], []
    for _ in range(3):
        dts.append(amr_step(o, m))
        refs.append(m.uold.copy())
    m.uold[:] = u0
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        for s in range(3):
            dt = gpu.coarse_step()
            assert dt == pytest.approx(dts[s], rel=1e-12)
            u = gpu.fetch_uold()
            err = rel_l1(u, refs[s])
            assert np.all(err <= TOL_FP64), (s, err)
            if spare:
                assert np.all(u[-spare:] == 7.0)
    finally:
        gpu.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
def test_amr_sedov_levels3to5_independent_runs_24_steps(prec):
    """The AMR Sedov on a small mesh: levels 3-5 refined by
    hydro_refine's 0.1 gradient criteria (outflow, gamma 1.4, moncen, HLLC,
    C = 0.8, interpol_type 1), 24 coarse steps with nsubcycle = 1.  The GPU
    (rh_coarse_step, its own courant_fine dt) and the oracle evolve
    independently; at every step the dt agrees to 1e-12 and the FP64 state
    to 1e-12 relative L1 per variable (FP32-bulk: density 1e-5), so the
    coarse-fine corrections and interpolated ghosts do not drift apart as
    they compound."""
    from ramses2_b200.mesh import sedov_amr_mesh

    m, g = sedov_amr_mesh(3, 5, radius=0.3)
    assert all(m.noct[l] for l in (3, 4, 5))
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                         interpol_type=1)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    dts, refs = [], []
    for _ in range(24):
        dts.append(amr_step(o, m))
        refs.append(m.uold.copy())
    m.uold[:] = u0
    gpu = GodunovGPU(m, P, precision=prec)
    try:
        for s in range(24):
            dt = gpu.coarse_step()
            err = rel_l1(gpu.fetch_uold(), refs[s])
            if prec == "fp64":
                assert dt == pytest.approx(dts[s], rel=1e-12), s
                assert np.all(err <= TOL_FP64), (s, err)
            else:
                assert dt == pytest.approx(dts[s], rel=1e-4), s
                assert err[0] <= TOL_FP32_RHO, (s, err)
    finally:
        gpu.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
def test_amr_deterministic_coarse_update_repeats_bitwise(prec):
    """rh_set_deterministic(1): the coarse-fine corrections go through
    per-face slots summed in a fixed order, so two AMR runs of four coarse
    steps are bitwise equal, and each stays within 1e-12 of the oracle (FP64;
    FP32-bulk: density 1e-5)."""
    m, P = amr_case("outflow", 1, 0)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    refs = []
    for _ in range(4):
        amr_step(o, m)
        refs.append(m.uold.copy())
    runs = []
    for _ in range(2):
        m.uold[:] = u0
        gpu = GodunovGPU(m, P, precision=prec, deterministic=True)
        try:
            states = []
            for s in range(4):
                gpu.coarse_step()
                states.append(gpu.fetch_uold())
                err = rel_l1(states[-1], refs[s])
                if prec == "fp64":
                    assert np.all(err <= TOL_FP64), (s, err)
                else:
                    assert err[0] <= TOL_FP32_RHO, (s, err)
        finally:
            gpu.close()
        runs.append(states)
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", ["fp64", "fp32_bulk"])
def test_amr_coarse_step_courant_values_match_a_fresh_courant_fine(prec):
    """After each concurrent coarse step every level's courant_fine values
    come from the step itself: the pencils' fused epilogue for the cells
    whose state they finish, and the coarse gather for the father cells it
    corrects afterwards.  They must equal a fresh courant_fine pass over the
    new state (parameters changed and restored so that nothing is reused):
    dt bitwise, the mass and energy sums to 1e-13."""
    from ramses2_b200.mesh import sedov_amr_mesh

    m, g = sedov_amr_mesh(3, 5, radius=0.3)
    levels = [l for l in range(m.levelmin, m.levelmax + 1) if m.noct[l]]
    assert len(levels) == 3
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                         interpol_type=1)
    gpu = GodunovGPU(m, P, precision=prec)
    try:
        for s in range(3):
            gpu.coarse_step()
            from_step = {l: gpu.courant_fine(l) for l in levels}
            fresh = {}
            for l in levels:
                gpu.params.courant_factor = 0.5
                gpu.courant_fine(l)
                gpu.params.courant_factor = 0.8
                fresh[l] = gpu.courant_fine(l)
            for l in levels:
                a, b = from_step[l], fresh[l]
                assert a[4] == b[4], (s, l, a, b)
                np.testing.assert_allclose(a[:3], b[:3], rtol=1e-13, err_msg="step %d level %d" % (s, l))
    finally:
        gpu.close()


@pytest.mark.parametrize("mesh_kind", ["amr", "uniform"])
def test_coarse_step_dt_after_leaf_calls_in_between(mesh_kind):
    """rh_coarse_step takes its dt from the courant_fine values the previous
    call left (copied to the host early).  Leaf calls between two coarse
    steps (a whole step through courant_fine / set_unew / godunov_fine /
    set_uold) write new values: the next coarse step must take the dt of the
    state they left, the one courant_fine now reports."""
    from ramses2_b200.mesh import sedov_amr_mesh

    if mesh_kind == "amr":
        m, g = sedov_amr_mesh(3, 5, radius=0.3)
    else:
        m = uniform_mesh(5, nsubgrid=1, bc="outflow")
        g = blast_state(m, 11, 1.4)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                         interpol_type=1)
    lev = [l for l in range(m.levelmin, m.levelmax + 1) if m.noct[l]]
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        for _ in range(2):
            gpu.coarse_step()
        before = min(min(m.dx(l) / P.smallc, gpu.courant_fine(l)[4]) for l in lev)
        amr_coarse_step(gpu, m)
        expect = min(min(m.dx(l) / P.smallc, gpu.courant_fine(l)[4]) for l in lev)
        assert expect != before
        assert gpu.coarse_step() == expect
    finally:
        gpu.close()


def test_amr_coarse_step_native_given_dt_fp32_bulk():
    """rh_coarse_step with the oracle's dt passed in (no courant_fine):
    FP32-bulk density within 1e-5 of the oracle's coarse step."""
    m, P = amr_case("outflow", 1, 0)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    dt = amr_step(o, m)
    ref = m.uold.copy()
    m.uold[:] = u0
    gpu = GodunovGPU(m, P, precision="fp32_bulk")
    try:
        assert gpu.coarse_step(dt) == dt
        err = rel_l1(gpu.fetch_uold(), ref)
    finally:
        gpu.close()
    assert err[0] <= TOL_FP32_RHO, err
    assert np.all(err <= 1e-4), err


def test_amr_step_fp32_bulk():
    m, P = amr_case("outflow", 1, 0)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    dt = amr_step(o, m)
    ref = m.uold.copy()
    m.uold[:] = u0
    gpu = GodunovGPU(m, P, precision="fp32_bulk")
    try:
        amr_step(gpu, m, dt)
        err = rel_l1(gpu.fetch_uold(), ref)
    finally:
        gpu.close()
    assert err[0] <= TOL_FP32_RHO, err
    assert np.all(err <= 1e-4), err


@pytest.mark.parametrize("ivar", [0, 1])
def test_upload_fine_matches_oracle_bitwise(ivar):
    """Restriction (hydro/upload.f90:74-271) of every level into its parent
    cells, FP64: bitwise equal to the oracle; FP32-bulk: within FP32 rounding."""
    m, P = amr_case("outflow", 1, ivar)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P, nthreads=1)
    lev = [l for l in range(m.levelmin, m.levelmax + 1) if m.noct[l]]
    for l in reversed(lev[:-1]):
        o.upload_fine(l)
    ref = m.uold.copy()
    assert not np.array_equal(ref, u0)
    for prec, tol in (("fp64", 0.0), ("fp32_bulk", 1e-6)):
        m.uold[:] = u0
        gpu = GodunovGPU(m, P, precision=prec)
        try:
            for l in reversed(lev[:-1]):
                gpu.upload_fine(l)
            out = gpu.fetch_uold()
        finally:
            gpu.close()
        if tol == 0.0:
            assert np.array_equal(out, ref)
        else:
            assert np.all(rel_l1(out, ref) <= tol), rel_l1(out, ref)


@pytest.mark.parametrize("case", ["amr", "outflow", "periodic", "reflexive"])
def test_hydro_flag_matches_oracle(case):
    """Gradient refinement flags (hydro_flag + hydro_refine): FP64 flags equal
    the oracle's cell for cell, including neighbours taken from parent cells
    across coarse-fine faces and from boundary ghosts; cells already flagged
    are not counted again."""
    from ramses2_b200._abi import FlagParams
    from ramses2_b200.mesh import sedov_amr_mesh

    if case == "amr":
        m, g = sedov_amr_mesh(4, 6, radius=0.25)
        F = FlagParams.make(err_grad_d=0.1, err_grad_p=0.1)
    else:
        m = uniform_mesh(5, nsubgrid=1, bc=case)
        g = blast_state(m, 21, 1.4)
        F = FlagParams.make(err_grad_d=0.2, err_grad_p=0.3, err_grad_u=0.5)
    P = HydroParams.make(gamma=g)
    lev = [l for l in range(m.levelmin, m.levelmax + 1) if m.noct[l]]
    o = oracle.OracleHydro(m, P)
    pre = np.zeros((m.ngridmax, 8), np.int32)
    pre[::7, 3] = 1
    ref, nref = pre.copy(), []
    for l in lev:
        nref.append(o.hydro_flag(l, F, ref))
    assert sum(nref) > 0
    for prec in ("fp64", "fp32_bulk"):
        gpu = GodunovGPU(m, P, precision=prec)
        try:
            out, nout = pre.copy(), []
            for l in lev:
                nout.append(gpu.hydro_flag(l, F, out))
        finally:
            gpu.close()
        if prec == "fp64":
            assert np.array_equal(out, ref)
            assert nout == nref
        else:
            assert np.mean(out != ref) <= 5e-3


def _tables_numpy(m, lev, txo, tyo, lz):
    """Pencil tables of a complete level, restated in numpy: pencils ordered
    (bz, by, bx); rows z = oz0-1 .. oz0+L; oct columns (y, x) of the tile
    plus one-oct halo; coordinates wrapped (periodic) or clamped."""
    n = [m.box_nx[d] << (lev - 1) for d in range(3)]
    idx = np.full(n[::-1], -1, dtype=np.int64)  # [z, y, x]
    g = m.grid[m.level_slice(lev)]
    ck = g["ckey"].astype(np.int64)
    idx[ck[:, 2], ck[:, 1], ck[:, 0]] = np.arange(len(g)) + m.head[lev] - 1

    def wc(v, nn, per):
        return v % nn if per else min(max(v, 0), nn - 1)

    hdr, tab = [], []
    for bz in range(-(-n[2] // lz)):
        for by in range(-(-n[1] // tyo)):
            for bx in range(-(-n[0] // txo)):
                L = min(lz, n[2] - bz * lz)
                hdr.append((bx * txo, by * tyo, bz * lz, L))
                for r in range(L + 2):
                    z = wc(bz * lz - 1 + r, n[2], m.periodic[2])
                    for j in range(tyo + 2):
                        y = wc(by * tyo - 1 + j, n[1], m.periodic[1])
                        for i in range(txo + 2):
                            tab.append(idx[z, y, wc(bx * txo - 1 + i, n[0], m.periodic[0])])
    return np.array(hdr), np.array(tab)


@pytest.mark.parametrize("bc,tile,box", [("outflow", (7, 7, 3), (1, 1, 1)), ("periodic", (8, 4, 5), (2, 1, 1)),
                                         (["periodic", "periodic", "outflow", "outflow", "reflexive", "reflexive"],
                                          (8, 8, 16), (1, 2, 1))])
def test_device_built_tables_match_restatement(bc, tile, box):
    """The device-side table builder of complete levels gives exactly the
    oct tables of the restated construction (wrap / clamp, pencil order)."""
    import ctypes as C

    from ramses2_b200._lib import lib

    m = uniform_mesh(4, nsubgrid=1, bc=bc, box_nx=box)
    sedov3d(m)
    P = HydroParams.make(gamma=1.4)
    gpu = GodunovGPU(m, P, tile=tile)
    try:
        gpu.step_uniform()  # builds the tables for the tile
        L = lib()
        npen, ntab = C.c_int(), C.c_longlong()
        assert L.rh_level_info(4, C.byref(npen), C.byref(ntab)) == 0
        hdr = np.zeros((npen.value, 4), np.int32)
        poff = np.zeros(npen.value, np.int64)
        tab = np.zeros(ntab.value, np.int32)
        assert L.rh_level_table(4, hdr.ctypes.data_as(C.POINTER(C.c_int)),
                                poff.ctypes.data_as(C.POINTER(C.c_longlong)),
                                tab.ctypes.data_as(C.POINTER(C.c_int)), ntab.value) == 0
    finally:
        gpu.close()
    want_hdr, want_tab = _tables_numpy(m, 4, tile[0], tile[1], tile[2])
    assert np.array_equal(hdr, want_hdr)
    assert np.array_equal(tab, want_tab)
    assert poff[0] == 0 and np.all(np.diff(poff) == (hdr[:-1, 3] + 2) * (tile[0] + 2) * (tile[1] + 2))
