"""The batch runtime (include/ramses_hydro_batch.h) against the FP64 oracle.

Every problem of a batch is the reference's single-level step on its own box
(hydro/umuscl.f90 unsplit + courant_fine dt, amr/amr_step.f90 order), so each
one must match the oracle run alone on a uniform mesh of the same box: FP64
relative L1 <= 1e-12 per conserved variable after several steps, FP32-bulk
density <= 1e-5 after one step.  A problem's result must not depend on what
else is in the batch (bitwise), and pool admission must follow the footprint.
"""
import os

import numpy as np
import pytest

import oracle
from ramses2_b200._abi import HydroParams
from ramses2_b200.batch import Batch, dense_to_octs, ic_blast, ic_host, ic_split, octs_to_dense, problem
from ramses2_b200.mesh import prim_to_cons, uniform_mesh

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32_RHO = 1e-5
NTHREADS = os.cpu_count() or 1


def rel_l1(a, b):
    num = np.abs(a - b).sum(axis=(1, 2, 3))
    den = np.abs(b).sum(axis=(1, 2, 3))
    return num / np.where(den > 0, den, 1.0)


def random_states(rng, g):
    out = []
    for _ in range(2):
        rho = 10 ** rng.uniform(-2, 2)
        p = 10 ** rng.uniform(-3, 1)
        cs = np.sqrt(g * p / rho)
        d = rng.standard_normal(3)
        d *= rng.uniform(0, 2) * cs / np.linalg.norm(d)
        out.append([rho, d[0], d[1], d[2], p])
    return out


def split_dense(n, axis, left, right, g):
    nx, ny, nz = n
    c = np.indices((nz, ny, nx))  # [z, y, x]
    coord = c[2 - axis]
    lm = coord < n[axis] // 2
    prims = [np.where(lm, left[v], right[v]).astype(np.float64) for v in range(5)]
    return prim_to_cons(*prims, g)


def blast_dense(n, dx, amb, p_in, radius, centre, g, ndim=3):
    nx, ny, nz = n
    z, y, x = np.indices((nz, ny, nx)).astype(np.float64)
    r2 = ((x + 0.5) * dx - centre[0]) ** 2 + ((y + 0.5) * dx - centre[1]) ** 2
    if ndim == 3:
        r2 = r2 + ((z + 0.5) * dx - centre[2]) ** 2
    inside = r2 <= radius * radius * (1 + 1e-12)
    prims = [np.full((nz, ny, nx), amb[v], np.float64) for v in range(5)]
    prims[4] = np.where(inside, p_in, amb[4])
    return prim_to_cons(*prims, g)


def oracle_run(dense, lev, box_nx, bc, P, nsteps):
    m = uniform_mesh(lev, nsubgrid=1, bc=bc, box_nx=box_nx)
    m.from_dense(dense, lev)
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    t = 0.0
    for _ in range(nsteps):
        dt, _ = o.step_uniform()
        t += dt
    return m.to_dense(m.uold, lev), t


# (cells, level, box_nx, bc, ic kind)
CASES = [
    ((16, 8, 8), 3, (2, 1, 1), "outflow", "split0"),
    ((8, 16, 8), 3, (1, 2, 1), "periodic", "blast"),
    ((8, 8, 16), 3, (1, 1, 2), "reflexive", "split2"),
    ((16, 16, 8), 3, (2, 2, 1), ["periodic", "periodic", "outflow", "outflow", "reflexive", "reflexive"], "host"),
    ((8, 8, 8), 3, (1, 1, 1), "outflow", "split1"),
]


def _make(case, rng, g):
    n, lev, bn, bc, kind = case
    dx = 1.0 / 2 ** lev
    if kind.startswith("split"):
        axis = int(kind[-1])
        left, right = random_states(rng, g)
        return split_dense(n, axis, left, right, g), ic_split(axis, left, right)
    if kind == "blast":
        amb = [1.0, 0.0, 0.0, 0.0, 1e-3]
        c = (n[0] * dx / 2, n[1] * dx / 2, n[2] * dx / 2)
        rad = 2.5 * dx
        return blast_dense(n, dx, amb, 50.0, rad, c, g), ic_blast(amb, 50.0, rad, c)
    # host: a random smooth state
    z, y, x = np.indices((n[2], n[1], n[0])) / 8.0
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.2 * np.sin(2 * np.pi * z)
    u = 0.3 * np.sin(2 * np.pi * y)
    v = -0.2 * np.cos(2 * np.pi * x)
    w = 0.1 * np.sin(2 * np.pi * (x + y))
    p = 1.0 + 0.3 * np.cos(2 * np.pi * z)
    dense = prim_to_cons(rho, u, v, w, p, g)
    return dense, ic_host(dense_to_octs(dense))


@pytest.mark.parametrize("riemann", ["llf", "hllc"])
def test_batch_fp64_matches_oracle_per_problem(riemann):
    rng = np.random.default_rng(7)
    g = 1.4
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann=riemann)
    nsteps = 3
    b = Batch("fp64", slope_type=2, riemann=riemann, pool_octs=1 << 14)
    try:
        ids, refs = [], []
        for case in CASES:
            n, lev, bn, bc, kind = case
            dense, ic = _make(case, rng, g)
            p = problem(n, dx=1.0 / 2 ** lev, bc=bc, gamma=g, courant_factor=0.8, max_steps=nsteps)
            ids.append(b.add(p, ic))
            refs.append(oracle_run(dense, lev, bn, bc, P, nsteps))
        b.step(nsteps + 2)  # extra steps must leave finished problems alone
        for pid, case, (ref, t_ref) in zip(ids, CASES, refs):
            st = b.status(pid)
            assert st["done"] and st["nstep"] == nsteps
            assert st["t"] == pytest.approx(t_ref, rel=1e-13)
            out = b.fetch_dense(pid)
            err = rel_l1(out, ref)
            assert np.all(err <= TOL_FP64), (case, err)
    finally:
        b.close()


def test_batch_fp32_bulk_one_step_density():
    rng = np.random.default_rng(3)
    g = 1.6
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    b = Batch("fp32_bulk", slope_type=2, riemann="hllc", pool_octs=1 << 14)
    try:
        for case in CASES:
            n, lev, bn, bc, kind = case
            dense, ic = _make(case, rng, g)
            pid = b.add(problem(n, dx=1.0 / 2 ** lev, bc=bc, gamma=g, courant_factor=0.8, max_steps=1), ic)
            ref, _ = oracle_run(dense, lev, bn, bc, P, 1)
            b.step(1)
            out = b.fetch_dense(pid)
            err = rel_l1(out, ref)
            assert err[0] <= TOL_FP32_RHO, (case, err)
            assert np.all(err <= 1e-4), (case, err)
            b.remove(pid)
    finally:
        b.close()


def _ensemble(rng, k):
    sizes = [8, 16, 24, 32]
    out = []
    for _ in range(k):
        n = tuple(int(rng.choice(sizes)) for _ in range(3))
        g = float(rng.uniform(1.1, 1.67))
        left, right = random_states(rng, g)
        axis = int(rng.integers(0, 3))
        p = problem(n, dx=1.0 / n[0], bc="outflow", gamma=g, courant_factor=0.6, max_steps=4)
        out.append((p, ic_split(axis, left, right)))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_batch_result_identical_alone_and_in_mix(precision):
    rng = np.random.default_rng(11)
    mix = _ensemble(rng, 24)
    target = mix[5]
    b = Batch(precision, pool_octs=1 << 16)
    try:
        pid = b.add(*target)
        b.step(4)
        alone = b.fetch(pid)
        st_alone = b.status(pid)
    finally:
        b.close()
    b = Batch(precision, pool_octs=1 << 16)
    try:
        ids = [b.add(p, ic) for p, ic in mix]
        b.step(3)
        # a late arrival joins mid-run; it must not disturb the others either
        late = b.add(*_ensemble(np.random.default_rng(99), 1)[0])
        b.step(3)
        mixed = b.fetch(ids[5])
        st_mix = b.status(ids[5])
        assert b.status(late)["nstep"] == 3
    finally:
        b.close()
    assert st_alone["nstep"] == st_mix["nstep"] == 4
    assert st_alone["t"] == st_mix["t"]
    assert np.array_equal(alone, mixed)


def test_batch_lands_on_t_end_and_stops():
    g = 1.4
    b = Batch("fp64", pool_octs=1 << 12)
    try:
        left, right = [1.0, 0, 0, 0, 1.0], [0.125, 0, 0, 0, 0.1]
        p = problem((32, 8, 8), dx=1.0 / 32, gamma=g, courant_factor=0.8, t_end=0.05)
        pid = b.add(p, ic_split(0, left, right))
        for _ in range(200):
            b.step(2)
            if b.status(pid)["done"]:
                break
        st = b.status(pid)
        assert st["done"]
        assert st["t"] == pytest.approx(0.05, rel=1e-12)
        u1 = b.fetch(pid)
        b.step(2)
        assert np.array_equal(u1, b.fetch(pid))
        # mass is conserved up to the outflow through the x faces, which is 0
        # while the waves are inside the box
        tot = st["totals"]
        assert tot[0] == pytest.approx((1.0 + 0.125) / 2 * 1.0 * 0.25 * 0.25, rel=1e-12)
    finally:
        b.close()


def test_batch_2d_problem_matches_oracle_plane():
    """A plane problem (ndim=2, one z oct layer, periodic z) is the 3D step of a
    z-uniform state with the 2-direction CFL dt (courant_fine ndim terms)."""
    rng = np.random.default_rng(5)
    g = 1.4
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    lev = 3
    dx = 1.0 / 2 ** lev
    left, right = random_states(rng, g)
    left[3] = right[3] = 0.0
    d3 = split_dense((16, 16, 8), 1, left, right, g)
    d2 = split_dense((16, 16, 2), 1, left, right, g)
    # 2-direction dt of the initial state
    dt = min(oracle.cmpdt(d2[:, z, y, x], dx, P, ndim=2)
             for z in range(2) for y in range(16) for x in range(16))
    dt = min(dt, dx / P.smallc)
    m = uniform_mesh(lev, nsubgrid=1, bc=["outflow"] * 4 + ["periodic"] * 2, box_nx=(2, 2, 1))
    m.from_dense(d3, lev)
    o = oracle.OracleHydro(m, P, nthreads=NTHREADS)
    o.step_uniform(dt)
    ref = m.to_dense(m.uold, lev)[:, :2]
    b = Batch("fp64", pool_octs=1 << 12)
    try:
        pid = b.add(problem((16, 16, 2), dx=dx, ndim=2, bc=["outflow"] * 4 + ["periodic"] * 2, gamma=g,
                            courant_factor=0.8, max_steps=1), ic_split(1, left, right))
        assert b.status(pid)["dt"] == pytest.approx(dt, rel=1e-14)
        b.step(1)
        out = b.fetch_dense(pid)
    finally:
        b.close()
    assert np.array_equal(out[:, 0], out[:, 1])
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err


def test_batch_pool_admission_and_reuse():
    b = Batch("fp32_bulk", pool_octs=3 * 512 + 64)
    try:
        p = problem((16, 16, 16), max_steps=1)  # 512 octs
        ic = ic_split(0, [1, 0, 0, 0, 1], [0.5, 0, 0, 0, 0.5])
        assert b.footprint(p) == 512 * (2 * 128 + 2 * 64)
        ids = [b.add(p, ic) for _ in range(3)]
        assert all(i is not None for i in ids)
        assert b.add(p, ic) is None  # RH_ENOMEM: the caller queues it
        b.remove(ids[1])
        again = b.add(p, ic)
        assert again is not None
        assert b.cells() == 3 * 4096
        b.step(1)
        assert b.cells() == 0
    finally:
        b.close()



@pytest.mark.parametrize("n,lev,box", [((2, 2, 2), 1, (1, 1, 1)), ((2, 16, 2), 1, (1, 8, 1)),
                                       ((30, 6, 10), 1, (15, 3, 5)), ((4, 4, 64), 1, (2, 2, 32))])
def test_batch_edge_shapes_match_oracle(n, lev, box):
    """Degenerate and ragged boxes (one oct, one-oct-thin, sizes that no tile
    divides, a pencil deeper than the tile): FP64 batch vs oracle, 2 steps."""
    rng = np.random.default_rng(sum(n))
    g = 1.4
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    dx = 1.0 / 2 ** lev
    z, y, x = np.indices((n[2], n[1], n[0]))
    rho = 1.0 + 0.5 * rng.random((n[2], n[1], n[0]))
    u = 0.3 * rng.standard_normal((n[2], n[1], n[0]))
    v = 0.3 * rng.standard_normal((n[2], n[1], n[0]))
    w = 0.3 * rng.standard_normal((n[2], n[1], n[0]))
    p = 1.0 + rng.random((n[2], n[1], n[0]))
    dense = prim_to_cons(rho, u, v, w, p, g)
    ref, t_ref = oracle_run(dense, lev, box, "outflow", P, 2)
    b = Batch("fp64", pool_octs=4096)
    try:
        pid = b.add(problem(n, dx=dx, bc="outflow", gamma=g, courant_factor=0.8, max_steps=2),
                    ic_host(dense_to_octs(dense)))
        b.step(2)
        out = b.fetch_dense(pid)
        assert b.status(pid)["t"] == pytest.approx(t_ref, rel=1e-13)
    finally:
        b.close()
    err = rel_l1(out, ref)
    assert np.all(err <= TOL_FP64), err


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
@pytest.mark.parametrize("slope,riemann", [(2, "hllc"), (1, "hll"), (0, "llf")])
def test_batch_plane_path_equals_pencil_path(precision, slope, riemann):
    """2D problems on the plane tile body give the pencil body's result bit for
    bit (its z slopes and z flux differences are exact zeros there): several
    boundary kinds, uneven sizes and tile-row counts (odd ones leave the last
    FP32-bulk tile pair half empty), a tall problem whose work items hold
    several tile bodies along y (the last item only part of a group), a 3D
    problem in the same batch, 6 steps."""
    cases = [((48, 32, 2), ["outflow"] * 4 + ["periodic"] * 2),
             ((16, 40, 2), ["reflexive", "outflow", "periodic", "periodic", "periodic", "periodic"]),
             ((30, 18, 2), ["reflexive"] * 4 + ["periodic"] * 2),
             ((24, 232, 2), ["outflow"] * 2 + ["periodic"] * 4)]
    results = {}
    for plane in (1, 0):
        b = Batch(precision, slope_type=slope, riemann=riemann, pool_octs=1 << 14)
        try:
            assert b.L.rh_batch_set_plane_path(plane) == 0
            ids = []
            for k, (n, bc) in enumerate(cases):
                st = random_states(np.random.default_rng(100 + k), 1.4)
                st[0][3] = st[1][3] = 0.0
                if k == 1:
                    ic = ic_blast([1.0, 0.0, 0.0, 0.0, 1e-3], 10.0, 0.15, [0.25, 0.6, 0.0])
                else:
                    ic = ic_split(k % 2, st[0], st[1])
                ids.append(b.add(problem(n, dx=1.0 / 64, ndim=2, bc=bc, gamma=1.4, max_steps=6), ic))
            ids.append(b.add(problem((16, 16, 16), max_steps=6), ic_split(2, [1, 0, 0, 0, 1], [0.1, 0, 0, 0, 0.1])))
            b.step(6)
            results[plane] = [(b.fetch(i), b.status(i)) for i in ids]
        finally:
            b.close()
    for (ua, sa), (ub, sb) in zip(results[1], results[0]):
        assert np.array_equal(ua, ub)
        assert sa["t"] == sb["t"] and sa["dt"] == sb["dt"] and sa["nstep"] == sb["nstep"] == 6
        # FP32-bulk plane items pair two tiles, so the partial sums group cells
        # differently: the totals agree to rounding, the states bit for bit
        assert sa["totals"] == pytest.approx(sb["totals"], rel=1e-12)
