"""Artificial diffusion (difmag > 0) in the CPU oracle: unsplit's cmpdivu and
cmpdiff (hydro/umuscl.f90:2392-2540, called at umuscl.f90:273-283).

The reference has no output for this option to pin to (its GPU and Metal
kernels have no artificial diffusion), so the oracle's loop-by-loop
restatement is checked against an independent vectorised statement of the
same formulas, and against the properties the formulas imply: nothing
happens in a fluid at rest, and the totals of a periodic box are
conserved."""
import numpy as np

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200.mesh import prim_to_cons, sedov3d, uniform_mesh


def _params(difmag, riemann="hllc"):
    return HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann=riemann, difmag=difmag)


def _random_block(nn, rng):
    """Conserved variables (5, nn+4, nn+4, nn+4) [var, k, j, i] of a random
    flow with compressing and expanding regions."""
    shape = (nn + 4,) * 3
    rho = 0.5 + rng.random(shape)
    u, v, w = (rng.normal(0.0, 0.7, shape) for _ in range(3))
    p = 0.3 + rng.random(shape)
    return np.ascontiguousarray(prim_to_cons(rho, u, v, w, p, 1.4))


def _diffusive_flux(uin, dx, dt, difmag, smallr):
    """cmpdivu + cmpdiff written with numpy over the whole block: the flux
    added to each face, shaped like oracle.unsplit's output
    (3, 5, nn+1, nn+1, nn+1) [dir, var, k, j, i], faces 1..nn+1 in Fortran
    indices.  Array index a holds Fortran index a - 1."""
    nn = uin.shape[-1] - 4
    r = np.maximum(uin[0], smallr)
    vel = [uin[1 + d] / r for d in range(3)]  # [k, j, i]
    f = nn + 1  # Fortran corners 1..nn+1 use cells 0..nn+1: array slices below
    sl = slice(2, 2 + f)  # cell i of corner i
    sm = slice(1, 1 + f)  # cell i-1 of corner i

    def q(c, kk, jj, ii):
        return vel[c][kk, jj, ii]

    fact = 0.25 / dx
    ux = fact * ((q(0, sl, sl, sl) - q(0, sl, sl, sm)) + (q(0, sl, sm, sl) - q(0, sl, sm, sm)) +
                 (q(0, sm, sl, sl) - q(0, sm, sl, sm)) + (q(0, sm, sm, sl) - q(0, sm, sm, sm)))
    vy = fact * ((q(1, sl, sl, sl) - q(1, sl, sm, sl)) + (q(1, sl, sl, sm) - q(1, sl, sm, sm)) +
                 (q(1, sm, sl, sl) - q(1, sm, sm, sl)) + (q(1, sm, sl, sm) - q(1, sm, sm, sm)))
    wz = fact * ((q(2, sl, sl, sl) - q(2, sm, sl, sl)) + (q(2, sl, sm, sl) - q(2, sm, sm, sl)) +
                 (q(2, sl, sl, sm) - q(2, sm, sl, sm)) + (q(2, sl, sm, sm) - q(2, sm, sm, sm)))
    div = ux + vy + wz  # corners [k, j, i] = Fortran (i, j, k), 1..nn+1
    out = np.zeros((3, 5, f, f, f))
    n = nn  # interior cells 1..nn -> corner-array index 0..nn-1
    # x faces: i = 1..nn+1, j, k = 1..nn; corners (i, j..j+1, k..k+1)
    d1 = 0.25 * (div[:n, :n, :] + div[:n, 1:n + 1, :] + div[1:n + 1, :n, :] + div[1:n + 1, 1:n + 1, :])
    du = uin[:, 2:2 + n, 2:2 + n, 2:2 + f] - uin[:, 2:2 + n, 2:2 + n, 1:1 + f]
    out[0, :, :n, :n, :] = dt * difmag * np.minimum(0.0, d1) * du
    # y faces: j = 1..nn+1, i, k = 1..nn; corners (i..i+1, j, k..k+1)
    d1 = 0.25 * (div[:n, :, :n] + div[:n, :, 1:n + 1] + div[1:n + 1, :, :n] + div[1:n + 1, :, 1:n + 1])
    du = uin[:, 2:2 + n, 2:2 + f, 2:2 + n] - uin[:, 2:2 + n, 1:1 + f, 2:2 + n]
    out[1, :, :n, :, :n] = dt * difmag * np.minimum(0.0, d1) * du
    # z faces: k = 1..nn+1, i, j = 1..nn; corners (i..i+1, j..j+1, k)
    d1 = 0.25 * (div[:, :n, :n] + div[:, :n, 1:n + 1] + div[:, 1:n + 1, :n] + div[:, 1:n + 1, 1:n + 1])
    du = uin[:, 2:2 + f, 2:2 + n, 2:2 + n] - uin[:, 1:1 + f, 2:2 + n, 2:2 + n]
    out[2, :, :, :n, :n] = dt * difmag * np.minimum(0.0, d1) * du
    return out


def test_diffusive_flux_matches_an_independent_statement():
    rng = np.random.default_rng(11)
    dx, dt, difmag = 1.0 / 32, 2e-3, 0.4
    for nn in (2, 4):
        uin = _random_block(nn, rng)
        f0 = oracle.unsplit(uin, dx, dt, _params(0.0))
        f1 = oracle.unsplit(uin, dx, dt, _params(difmag))
        want = _diffusive_flux(uin, dx, dt, difmag, _params(0.0).smallr)
        got = f1 - f0
        scale = np.abs(f0).max() + np.abs(want).max()
        assert np.abs(want).max() > 1e-3 * np.abs(f0).max()  # the test flow does compress
        assert np.abs(got - want).max() <= 1e-14 * scale, np.abs(got - want).max() / scale


def test_no_diffusion_in_a_fluid_at_rest():
    # Sedov's initial state is at rest: every corner divergence is exactly 0
    # and the first step is the one without diffusion, bit for bit
    states = []
    for difmag in (0.0, 0.5):
        m = uniform_mesh(4, nsubgrid=1, bc="outflow")
        sedov3d(m)
        o = oracle.OracleHydro(m, _params(difmag))
        o.step_uniform()
        states.append(m.uold.copy())
        o.step_uniform()  # the blast now moves: diffusion acts
        states.append(m.uold.copy())
    assert np.array_equal(states[0], states[2])
    assert not np.array_equal(states[1], states[3])


def test_diffusion_conserves_a_periodic_box():
    m = uniform_mesh(4, nsubgrid=1, bc="periodic")
    rng = np.random.default_rng(5)
    lev = 4
    shape = m.uold[m.level_slice(lev)].shape[::2]
    rho = 1 + 0.5 * rng.random(shape)
    u, v, w = (rng.normal(0, 0.5, shape) for _ in range(3))
    p = 0.5 + rng.random(shape)
    m.uold[m.level_slice(lev)] = np.transpose(prim_to_cons(rho, u, v, w, p, 1.4), (1, 0, 2))
    ref = m.uold.copy()
    tot0 = m.uold.sum(axis=(0, 2))
    o = oracle.OracleHydro(m, _params(0.3))
    dts = [o.step_uniform()[0] for _ in range(4)]
    tot = m.uold.sum(axis=(0, 2))
    scale = np.abs(m.uold).sum(axis=(0, 2))
    assert np.all(np.abs(tot - tot0) <= 1e-13 * scale), (tot - tot0) / scale
    # the same steps without diffusion end elsewhere
    with_diffusion = m.uold.copy()
    m.uold[:] = ref
    o = oracle.OracleHydro(m, _params(0.0))
    for dt in dts:
        o.step_uniform(dt)
    rel = np.abs(with_diffusion - m.uold).max() / np.abs(m.uold).max()
    assert rel > 1e-6, rel
