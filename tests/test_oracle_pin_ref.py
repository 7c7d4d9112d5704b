"""Pins the FP64 oracle to the reference's own code.

The reference's hydro path is Fortran (no compiler here), but it also ships a
Metal port of its GPU kernel (metal/kernels/hydro.metal, float32, mirroring
gpu/gpu_hydro.cuf).  oracle/Makefile compiles that shader source as C++ from
the reference checkout (target `ref`, stand-in MSL headers in oracle/msl_shim)
into oracle/_ref/librh_ref_msl.so.  These tests feed identical inputs to the
shader functions and to the oracle and require agreement at FP32 rounding:
the three Riemann solvers, the per-oct trace + Riemann pipeline (ctoprim,
slopes with the momentum bound, Hancock predictor, face states, rotations)
for every slope type, the courant_fine reduction a whole Godunov step of a periodic level
(the shader's hydro_integrator_kernel: gather, trace, Riemann, conservative
update), the restriction (upload_kernel) and the gradient flags
(flag.metal's hydro_flag_kernel).

The same shader source is also built with its arithmetic in FP64
(oracle/_ref/librh_ref_msl64.so; msl_shim turns the shader's float into
double), and the *_fp64 tests require agreement within 1e-12: measured here,
the Riemann fluxes agree to 4e-15 of the largest flux, an oct's face fluxes
to 1.3e-15 and a whole Godunov step to 1e-16 relative L1 per variable, so the
oracle (and through it the CUDA path, 1e-12 from the oracle) follows the
reference's own algorithm at FP64 rounding.  Skipped where the shader
libraries were not built (no reference checkout)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200.mesh import prim_to_cons, riemann3d_state, uniform_mesh

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "librh_ref_msl.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference shader library not built")


def _lib():
    L = C.CDLL(REF)
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C")
    L.ref_msl_riemann.argtypes = [C.c_int, f32, f32, C.c_float, C.c_float, C.c_float, C.c_float, f32]
    L.ref_msl_oct_fluxes.argtypes = [f32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
                                     f32]
    L.ref_msl_cmpdt.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                C.c_float, C.c_float, C.c_void_p, C.c_void_p]
    L.ref_msl_godunov.argtypes = [C.c_void_p] * 4 + [C.c_int] * 6 + [C.c_float] * 5 + [C.c_int, C.c_int,
                                                                                       C.c_void_p, C.c_float]
    L.ref_msl_upload.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [C.c_float] * 3
    L.ref_msl_hydro_flag.argtypes = [C.c_void_p] * 3 + [C.c_int] * 2 + [C.c_float] * 7
    return L


def _nbor27(m, no):
    """The shader's neighbour table of a periodic complete level: 1-based
    index of each of the 27 octs around an oct (x fastest)."""
    ck = m.grid["ckey"].astype(np.int64)
    idx = np.zeros((no, no, no), np.int64)
    idx[ck[:, 0], ck[:, 1], ck[:, 2]] = np.arange(len(ck)) + 1
    nbor = np.zeros((len(ck), 27), np.int32)
    for t in range(27):
        d = (t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1)
        nbor[:, t] = idx[(ck[:, 0] + d[0]) % no, (ck[:, 1] + d[1]) % no, (ck[:, 2] + d[2]) % no]
    return nbor


def _f32exact(a):
    """Round to float32 and back, so both sides see the same inputs."""
    return np.asarray(a, np.float32).astype(np.float64)


@pytest.mark.parametrize("solver", [1, 2, 3])
def test_riemann_solvers_match_reference_shader(solver):
    L = _lib()
    rng = np.random.default_rng(solver)
    g = 1.4
    P = HydroParams.make(gamma=g, smallr=1e-10, smallc=1e-10)
    worst = 0.0
    for _ in range(2000):
        q = []
        for _ in range(2):
            rho = 10 ** rng.uniform(-2, 2)
            p = 10 ** rng.uniform(-3, 2)
            c = np.sqrt(g * p / rho)
            q.append(_f32exact([rho, *(rng.uniform(-3, 3, 3) * c), p]))
        smax = float(np.float32(10 ** rng.uniform(0, 2)))
        ref = oracle.riemann(solver, q[0], q[1], P, smax_cap=smax)[:5]
        out = np.zeros(5, np.float32)
        L.ref_msl_riemann(solver, q[0].astype(np.float32), q[1].astype(np.float32), g, 1e-10, 1e-20, smax, out)
        scale = np.abs(ref).max()
        worst = max(worst, float(np.abs(out - ref).max() / scale))
    assert worst <= 2e-5, worst


@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc"])
@pytest.mark.parametrize("slope", [0, 1, 2])
def test_oct_fluxes_match_reference_shader(riemann, slope):
    """unsplit on one oct's 6^3 stencil vs the shader's trace_3d +
    riemann_driver: every face flux of the oct, each direction."""
    L = _lib()
    rng = np.random.default_rng(10 * slope + len(riemann))
    g, dx, dt, cour = 1.4, 0.1, 0.01, 0.8
    rid = {"llf": 1, "hll": 2, "hllc": 3}[riemann]
    P = HydroParams.make(gamma=g, courant_factor=cour, slope_type=slope, riemann=riemann)
    worst = 0.0
    for _ in range(40):
        rho = rng.uniform(0.5, 2.0, (6, 6, 6))
        p = rng.uniform(0.5, 2.0, (6, 6, 6))
        u, v, w = (rng.uniform(-0.5, 0.5, (6, 6, 6)) for _ in range(3))
        cons = _f32exact(prim_to_cons(rho, u, v, w, p, g))  # (5, k, j, i)
        fo = oracle.unsplit(cons, dx, dt, P) / (dt / dx)   # [dim][var][k][j][i]
        out = np.zeros(180, np.float32)
        L.ref_msl_oct_fluxes(np.ascontiguousarray(cons, np.float32), g, 1e-10, 1e-20, dt / dx, cour * dx / dt,
                             slope, rid, out)
        pairs = [(out[:60].reshape(5, 2, 2, 3), fo[0][:, 0:2, 0:2, 0:3]),
                 (out[60:120].reshape(5, 2, 3, 2), fo[1][:, 0:2, 0:3, 0:2]),
                 (out[120:].reshape(5, 3, 2, 2), fo[2][:, 0:3, 0:2, 0:2])]
        for a, b in pairs:
            err = np.abs(a - b).max(axis=(1, 2, 3)) / np.abs(b).max(axis=(1, 2, 3))
            worst = max(worst, float(err.max()))
    assert worst <= 2e-6, worst


def test_courant_fine_matches_reference_shader():
    L = _lib()
    m = uniform_mesh(4, bc="outflow", gravity=(0.2, -0.1, 0.3))
    g, dense = riemann3d_state(np.random.default_rng(1), 16, gamma=1.4)
    m.from_dense(dense, 4)
    m.uold[:] = _f32exact(m.uold)
    P = HydroParams.make(gamma=g, courant_factor=0.8)
    ref = oracle.OracleHydro(m, P).courant_fine(4)
    u32 = np.ascontiguousarray(m.uold, np.float32)
    grav = np.array(m.gravity, np.float32)
    out = np.zeros(5, np.float32)
    L.ref_msl_cmpdt(m.grid.ctypes.data, u32.ctypes.data, 1, int(m.noct[4]), m.dx(4), g, P.smallr, P.smallc ** 2,
                    0.8, grav.ctypes.data, out.ctypes.data)
    assert out[4] == pytest.approx(ref[4], rel=1e-6)   # dt
    assert out[0] == pytest.approx(ref[0], rel=2e-4)   # mass (float32 running sum of 32768 cells)
    assert out[1] == pytest.approx(ref[1], rel=2e-4)   # total energy


@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc"])
@pytest.mark.parametrize("slope", [0, 1, 2])
def test_godunov_step_matches_reference_shader(riemann, slope):
    """One step of a periodic 16^3 level: oracle godunov_fine (FP64) vs the
    shader's hydro_integrator_kernel (float32; one threadgroup per oct run by
    one thread) fed the same float32-representable state and the shader's
    27-neighbour table.  The new state agrees to float32 storage rounding and
    the update (unew - uold) to float32 arithmetic."""
    L = _lib()
    lev, n, no, g = 4, 16, 8, 1.4
    m = uniform_mesh(lev, bc="periodic")
    zz, yy, xx = (np.indices((n, n, n)) + 0.5) / n
    rho = 1 + 0.3 * np.sin(2 * np.pi * xx) * np.cos(2 * np.pi * yy) + 0.2 * np.sin(2 * np.pi * zz)
    p = 1 + 0.5 * np.cos(2 * np.pi * (xx - zz))
    m.from_dense(prim_to_cons(rho, 0.4 * np.sin(2 * np.pi * yy), -0.3 * np.cos(2 * np.pi * zz),
                              0.2 * np.sin(2 * np.pi * (xx + yy)), p, g), lev)
    m.uold[:] = _f32exact(m.uold)
    ck = m.grid["ckey"]
    nbor = _nbor27(m, no)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=slope, riemann=riemann)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P)
    dt = float(np.float32(0.5 * o.courant_fine(lev)[4]))
    o.set_unew(lev)
    o.godunov_fine(lev, dt)
    ref = o.unew.copy()
    u32 = np.ascontiguousarray(u0, np.float32)
    un32 = u32.copy()
    grav = np.zeros(3, np.float32)
    dx = m.dx(lev)
    L.ref_msl_godunov(m.grid.ctypes.data, u32.ctypes.data, un32.ctypes.data, nbor.ctypes.data, 1, len(ck), len(ck),
                      lev, lev, lev, g, P.smallr, P.smallc ** 2, dt, dx, slope, {"llf": 1, "hll": 2, "hllc": 3}[riemann],
                      grav.ctypes.data, 0.8 * dx / dt)
    out = un32.astype(np.float64)
    state = np.abs(out - ref).sum(axis=(0, 2)) / np.abs(ref).sum(axis=(0, 2))
    update = np.abs(out - ref).sum(axis=(0, 2)) / np.abs(ref - u0).sum(axis=(0, 2))
    assert np.all(state <= 2e-7), state
    assert np.all(update <= 1e-4), update


def test_hydro_flags_match_reference_shader():
    """Gradient flags of a periodic level (every neighbour exists, where the
    CPU and GPU reference flaggers coincide): same cells flagged."""
    from ramses2_b200._abi import FlagParams

    L = _lib()
    rng = np.random.default_rng(21)
    m = uniform_mesh(5, bc="periodic")
    g, dense = riemann3d_state(rng, 32, gamma=1.4)
    zz, yy, xx = (np.indices((32, 32, 32)) + 0.5) / 32
    dense[0] *= 1 + 0.3 * np.sin(4 * np.pi * xx) * np.cos(2 * np.pi * yy) + 0.1 * zz
    m.from_dense(dense, 5)
    m.uold[:] = _f32exact(m.uold)
    P = HydroParams.make(gamma=g)
    ref = np.zeros((m.ngridmax, 8), np.int32)
    n = oracle.OracleHydro(m, P).hydro_flag(5, FlagParams.make(err_grad_d=0.2, err_grad_p=0.3), ref)
    out = np.zeros((m.ngridmax, 8), np.int32)
    u32 = np.ascontiguousarray(m.uold, np.float32)
    L.ref_msl_hydro_flag(out.ctypes.data, _nbor27(m, 16).ctypes.data, u32.ctypes.data, 1, int(m.noct[5]), g,
                         P.smallr, P.smallc ** 2, 0.2, 0.3, 1e-10, 1e-10)
    assert n > 0 and np.array_equal(out, ref)


@pytest.mark.parametrize("ivar", [0, 1])
def test_upload_matches_reference_shader(ivar):
    from ramses2_b200.mesh import amr_mesh, fill_amr_prim

    L = _lib()
    m = amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.52) ** 2).sum(-1)) < 0.16)

    def prim(x, l):
        r = np.sqrt(((x - 0.5) ** 2).sum(-1))
        z = np.zeros_like(r)
        return (1 + 0.5 * np.exp(-r ** 2 / 0.01), 0.3 + 0.2 * np.sin(6 * x[..., 1]), -0.2 + z, 0.1 + 0.1 * x[..., 0],
                1 + 4 * np.exp(-r ** 2 / 0.004))

    fill_amr_prim(m, prim, 1.4)
    m.uold[:] = _f32exact(m.uold)
    P = HydroParams.make(gamma=1.4, interpol_var=ivar)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P)
    for lev in (5, 4):
        o.upload_fine(lev)
    ref = m.uold.copy()
    key = {(int(r["lev"]), *map(int, r["ckey"])): i + 1 for i, r in enumerate(m.grid)}
    father = np.array([key.get((int(r["lev"]) - 1, *(int(c) // 2 for c in r["ckey"])), 0) for r in m.grid], np.int32)
    u32 = np.ascontiguousarray(u0, np.float32)
    for lev in (6, 5):
        L.ref_msl_upload(m.grid.ctypes.data, father.ctypes.data, u32.ctypes.data, int(m.head[lev]), int(m.noct[lev]),
                         ivar, 1.4, P.smallr, P.smallc ** 2)
    assert np.abs(u32 - ref).max() <= 2e-7 * np.abs(ref).max()


# ---------------------------------------------------------------------------
# The same shader source built with its arithmetic in FP64
# (oracle/_ref/librh_ref_msl64.so, msl_shim's RH_MSL_DOUBLE): the oracle must
# agree with the reference's own algorithm at FP64 rounding, not FP32.
# ---------------------------------------------------------------------------
REF64 = REF.replace("librh_ref_msl.so", "librh_ref_msl64.so")
needs64 = pytest.mark.skipif(not os.path.exists(REF64), reason="FP64 shader library not built")


def _lib64():
    L = C.CDLL(REF64)
    f64 = np.ctypeslib.ndpointer(np.float64, flags="C")
    d = C.c_double
    L.ref_msl_riemann.argtypes = [C.c_int, f64, f64, d, d, d, d, f64]
    L.ref_msl_oct_fluxes.argtypes = [f64, d, d, d, d, d, C.c_int, C.c_int, f64]
    L.ref_msl_cmpdt.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, d, d, d, d, d, C.c_void_p, C.c_void_p]
    L.ref_msl_godunov.argtypes = [C.c_void_p] * 4 + [C.c_int] * 6 + [d] * 5 + [C.c_int, C.c_int, C.c_void_p, d]
    L.ref_msl_upload.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [d] * 3
    L.ref_msl_hydro_flag.argtypes = [C.c_void_p] * 3 + [C.c_int] * 2 + [d] * 7
    return L


@needs64
@pytest.mark.parametrize("solver", [1, 2, 3])
def test_riemann_solvers_match_reference_shader_fp64(solver):
    """2,000 wide-range state pairs per solver (density 1e-2..1e2, pressure
    1e-3..1e2, velocities up to 3 sound speeds, random smax cap): every flux
    component within 1e-12 of the largest one."""
    L = _lib64()
    rng = np.random.default_rng(100 + solver)
    g = 1.4
    P = HydroParams.make(gamma=g, smallr=1e-10, smallc=1e-10)
    worst = 0.0
    for _ in range(2000):
        q = []
        for _ in range(2):
            rho = 10 ** rng.uniform(-2, 2)
            p = 10 ** rng.uniform(-3, 2)
            c = np.sqrt(g * p / rho)
            q.append(np.array([rho, *(rng.uniform(-3, 3, 3) * c), p]))
        smax = 10 ** rng.uniform(0, 2)
        ref = oracle.riemann(solver, q[0], q[1], P, smax_cap=smax)[:5]
        out = np.zeros(5)
        L.ref_msl_riemann(solver, q[0], q[1], g, 1e-10, 1e-20, smax, out)
        worst = max(worst, float(np.abs(out - ref).max() / np.abs(ref).max()))
    assert worst <= 1e-12, worst


@needs64
@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc"])
@pytest.mark.parametrize("slope", [0, 1, 2])
def test_oct_fluxes_match_reference_shader_fp64(riemann, slope):
    """Every face flux of an oct from a random 6^3 stencil (ctoprim, slopes
    with the momentum bound, Hancock predictor, rotations, Riemann solver):
    within 1e-12 of the largest flux of its variable and direction."""
    L = _lib64()
    rng = np.random.default_rng(200 + 10 * slope + len(riemann))
    g, dx, dt, cour = 1.4, 0.1, 0.01, 0.8
    rid = {"llf": 1, "hll": 2, "hllc": 3}[riemann]
    P = HydroParams.make(gamma=g, courant_factor=cour, slope_type=slope, riemann=riemann)
    worst = 0.0
    for _ in range(40):
        rho = rng.uniform(0.5, 2.0, (6, 6, 6))
        p = rng.uniform(0.5, 2.0, (6, 6, 6))
        u, v, w = (rng.uniform(-0.5, 0.5, (6, 6, 6)) for _ in range(3))
        cons = np.ascontiguousarray(prim_to_cons(rho, u, v, w, p, g))
        fo = oracle.unsplit(cons, dx, dt, P) / (dt / dx)
        out = np.zeros(180)
        L.ref_msl_oct_fluxes(cons, g, 1e-10, 1e-20, dt / dx, cour * dx / dt, slope, rid, out)
        pairs = [(out[:60].reshape(5, 2, 2, 3), fo[0][:, 0:2, 0:2, 0:3]),
                 (out[60:120].reshape(5, 2, 3, 2), fo[1][:, 0:2, 0:3, 0:2]),
                 (out[120:].reshape(5, 3, 2, 2), fo[2][:, 0:3, 0:2, 0:2])]
        for a, b in pairs:
            err = np.abs(a - b).max(axis=(1, 2, 3)) / np.abs(b).max(axis=(1, 2, 3))
            worst = max(worst, float(err.max()))
    assert worst <= 1e-12, worst


@needs64
def test_courant_fine_matches_reference_shader_fp64():
    """courant_fine of a 16^3 level with constant gravity: dt within 1e-12
    (the shader's 0.0001f gravity floor differs from 1e-4 by 2.5e-12, which
    moves dt by less), mass and total energy within 1e-12 (the shader adds
    per-cell values in another order)."""
    L = _lib64()
    m = uniform_mesh(4, bc="outflow", gravity=(0.2, -0.1, 0.3))
    g, dense = riemann3d_state(np.random.default_rng(1), 16, gamma=1.4)
    m.from_dense(dense, 4)
    P = HydroParams.make(gamma=g, courant_factor=0.8)
    ref = oracle.OracleHydro(m, P).courant_fine(4)
    u = np.ascontiguousarray(m.uold)
    grav = np.array(m.gravity, np.float64)
    out = np.zeros(5)
    L.ref_msl_cmpdt(m.grid.ctypes.data, u.ctypes.data, 1, int(m.noct[4]), m.dx(4), g, P.smallr, P.smallc ** 2,
                    0.8, grav.ctypes.data, out.ctypes.data)
    assert out[4] == pytest.approx(ref[4], rel=1e-12)
    assert out[0] == pytest.approx(ref[0], rel=1e-12)
    assert out[1] == pytest.approx(ref[1], rel=1e-12)


@needs64
@pytest.mark.parametrize("riemann", ["llf", "hll", "hllc"])
@pytest.mark.parametrize("slope", [0, 1, 2])
def test_godunov_step_matches_reference_shader_fp64(riemann, slope):
    """A whole Godunov step of a periodic 16^3 level through the shader's
    hydro_integrator_kernel in FP64 against the oracle's godunov_fine.

    The two restate different reference files: the oracle follows the CPU
    path (hydro/umuscl.f90 + godunov_fine.f90), the shader the GPU kernel
    (gpu/gpu_hydro.cuf).  Where their operation orders differ:
      * face fluxes: the CPU path scales each flux by dt/dx inside cmpflxm
        (umuscl.f90:1472-1607) and adds flux(i) - flux(i+1) to unew
        (godunov_fine.f90:733-816); the GPU path keeps unscaled fluxes and
        adds dtdx * (F_left - F_right) per cell (gpu/gpu_hydro.cuf:3887-3912);
      * the trace's source terms and the slope products group their
        additions differently.
    Each is one or two roundings of a term of the update, so the update
    (unew - uold) agrees to a few ulps of the largest flux difference: bound
    1e-12 relative L1 on the update, 1e-14 on the state."""
    L = _lib64()
    lev, n, no, g = 4, 16, 8, 1.4
    m = uniform_mesh(lev, bc="periodic")
    zz, yy, xx = (np.indices((n, n, n)) + 0.5) / n
    rho = 1 + 0.3 * np.sin(2 * np.pi * xx) * np.cos(2 * np.pi * yy) + 0.2 * np.sin(2 * np.pi * zz)
    p = 1 + 0.5 * np.cos(2 * np.pi * (xx - zz))
    m.from_dense(prim_to_cons(rho, 0.4 * np.sin(2 * np.pi * yy), -0.3 * np.cos(2 * np.pi * zz),
                              0.2 * np.sin(2 * np.pi * (xx + yy)), p, g), lev)
    ck = m.grid["ckey"]
    nbor = _nbor27(m, no)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=slope, riemann=riemann)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P)
    dt = 0.5 * o.courant_fine(lev)[4]
    o.set_unew(lev)
    o.godunov_fine(lev, dt)
    ref = o.unew.copy()
    u = np.ascontiguousarray(u0)
    un = u.copy()
    grav = np.zeros(3)
    dx = m.dx(lev)
    L.ref_msl_godunov(m.grid.ctypes.data, u.ctypes.data, un.ctypes.data, nbor.ctypes.data, 1, len(ck), len(ck),
                      lev, lev, lev, g, P.smallr, P.smallc ** 2, dt, dx, slope, {"llf": 1, "hll": 2, "hllc": 3}[riemann],
                      grav.ctypes.data, 0.8 * dx / dt)
    state = np.abs(un - ref).sum(axis=(0, 2)) / np.abs(ref).sum(axis=(0, 2))
    update = np.abs(un - ref).sum(axis=(0, 2)) / np.abs(ref - u0).sum(axis=(0, 2))
    assert np.all(state <= 1e-14), state
    assert np.all(update <= 1e-12), update


@needs64
def test_hydro_flags_match_reference_shader_fp64():
    from ramses2_b200._abi import FlagParams

    L = _lib64()
    rng = np.random.default_rng(21)
    m = uniform_mesh(5, bc="periodic")
    g, dense = riemann3d_state(rng, 32, gamma=1.4)
    zz, yy, xx = (np.indices((32, 32, 32)) + 0.5) / 32
    dense[0] *= 1 + 0.3 * np.sin(4 * np.pi * xx) * np.cos(2 * np.pi * yy) + 0.1 * zz
    m.from_dense(dense, 5)
    P = HydroParams.make(gamma=g)
    ref = np.zeros((m.ngridmax, 8), np.int32)
    nref = oracle.OracleHydro(m, P).hydro_flag(5, FlagParams.make(err_grad_d=0.2, err_grad_p=0.3), ref)
    out = np.zeros((m.ngridmax, 8), np.int32)
    u = np.ascontiguousarray(m.uold)
    L.ref_msl_hydro_flag(out.ctypes.data, _nbor27(m, 16).ctypes.data, u.ctypes.data, 1, int(m.noct[5]), g,
                         P.smallr, P.smallc ** 2, 0.2, 0.3, 1e-10, 1e-10)
    assert nref > 0 and np.array_equal(out, ref)


@needs64
@pytest.mark.parametrize("ivar", [0, 1])
def test_upload_matches_reference_shader_fp64(ivar):
    from ramses2_b200.mesh import amr_mesh, fill_amr_prim

    L = _lib64()
    m = amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.52) ** 2).sum(-1)) < 0.16)

    def prim(x, l):
        r = np.sqrt(((x - 0.5) ** 2).sum(-1))
        z = np.zeros_like(r)
        return (1 + 0.5 * np.exp(-r ** 2 / 0.01), 0.3 + 0.2 * np.sin(6 * x[..., 1]), -0.2 + z, 0.1 + 0.1 * x[..., 0],
                1 + 4 * np.exp(-r ** 2 / 0.004))

    fill_amr_prim(m, prim, 1.4)
    P = HydroParams.make(gamma=1.4, interpol_var=ivar)
    u0 = m.uold.copy()
    o = oracle.OracleHydro(m, P)
    for lev in (5, 4):
        o.upload_fine(lev)
    ref = m.uold.copy()
    key = {(int(r["lev"]), *map(int, r["ckey"])): i + 1 for i, r in enumerate(m.grid)}
    father = np.array([key.get((int(r["lev"]) - 1, *(int(c) // 2 for c in r["ckey"])), 0) for r in m.grid], np.int32)
    u = np.ascontiguousarray(u0)
    for lev in (6, 5):
        L.ref_msl_upload(m.grid.ctypes.data, father.ctypes.data, u.ctypes.data, int(m.head[lev]), int(m.noct[lev]),
                         ivar, 1.4, P.smallr, P.smallc ** 2)
    assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()
