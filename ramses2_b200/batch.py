"""Many independent uniform-grid hydro problems on one B200 (the batch ABI,
include/ramses_hydro_batch.h).

Each problem is the reference's single-level step (hydro/umuscl.f90 unsplit
MUSCL-Hancock + courant_fine dt, amr/amr_step.f90 order) on its own box with its
own CFL dt; problems of uneven sizes share one device pool and advance together
in one persistent kernel launch per step.  States are exchanged in the
reference's per-oct layout (noct, 5, 8) with octs in row-major order
(oct = (z*nyo + y)*nxo + x); :func:`dense_to_octs` / :func:`octs_to_dense`
convert from/to dense (5, nz, ny, nx) arrays.
"""
import ctypes as C

import numpy as np

from ._abi import (RH_IC_BLAST, RH_IC_HOST, RH_IC_SPLIT, RH_PREC_FP32_BULK, RH_PREC_FP64, RH_RIEMANN, BatchIC,
                   BatchProblem, dptr)
from ._lib import check, lib
from .mesh import BC_NAMES

PRECISION = {"fp64": RH_PREC_FP64, "fp32_bulk": RH_PREC_FP32_BULK, "fp32": RH_PREC_FP32_BULK}
RH_ENOMEM = 2


def dense_to_octs(dense):
    """(5, nz, ny, nx) -> (noct, 5, 8), octs row-major, cells x fastest."""
    v, nz, ny, nx = dense.shape
    a = dense.reshape(v, nz // 2, 2, ny // 2, 2, nx // 2, 2)
    # -> [oz, oy, ox, var, cz, cy, cx]
    a = a.transpose(1, 3, 5, 0, 2, 4, 6)
    return np.ascontiguousarray(a.reshape(-1, v, 8))


def octs_to_dense(octs, n):
    """(noct, 5, 8) row-major octs -> (5, nz, ny, nx) for a box of n = (nx, ny, nz) cells."""
    nx, ny, nz = n
    a = octs.reshape(nz // 2, ny // 2, nx // 2, 5, 2, 2, 2)
    a = a.transpose(3, 0, 4, 1, 5, 2, 6)
    return np.ascontiguousarray(a.reshape(5, nz, ny, nx))


def problem(n, dx=None, ndim=3, bc="outflow", gamma=1.4, smallr=1e-10, smallc=1e-10, courant_factor=0.8,
            t_end=0.0, max_steps=0):
    """An rh_batch_problem; dx defaults to 1/n[0] (unit box in x)."""
    p = BatchProblem()
    for d in range(3):
        p.n[d] = int(n[d])
    p.ndim = int(ndim)
    bcs = [bc] * 6 if isinstance(bc, (str, int)) else list(bc)
    for i in range(6):
        p.bound_type[i] = BC_NAMES[bcs[i]] if isinstance(bcs[i], str) else int(bcs[i])
    p.dx = float(dx if dx is not None else 1.0 / n[0])
    p.gamma, p.smallr, p.smallc, p.courant_factor = float(gamma), float(smallr), float(smallc), float(courant_factor)
    p.t_end = float(t_end)
    p.max_steps = int(max_steps)
    return p


def ic_split(axis, left, right):
    """Two primitive states (rho, u, v, w, p) split at the middle of ``axis``."""
    ic = BatchIC()
    ic.kind = RH_IC_SPLIT
    ic.axis = int(axis)
    for v in range(5):
        ic.left[v] = float(left[v])
        ic.right[v] = float(right[v])
    return ic


def ic_blast(ambient, p_in, radius, centre):
    """Uniform primitive state with pressure p_in inside a sphere (disc in 2D)."""
    ic = BatchIC()
    ic.kind = RH_IC_BLAST
    for v in range(5):
        ic.ambient[v] = float(ambient[v])
    ic.p_in = float(p_in)
    ic.radius = float(radius)
    for d in range(3):
        ic.centre[d] = float(centre[d])
    return ic


def ic_host(octs):
    """Conserved state (noct, 5, 8) copied from the host (kept alive by the IC)."""
    ic = BatchIC()
    ic.kind = RH_IC_HOST
    a = np.ascontiguousarray(octs, np.float64)
    ic.host_uold = a.ctypes.data
    ic._keep = a
    return ic


class Batch:
    """The process's batch (one per process; rh_init must have run)."""

    def __init__(self, precision="fp64", slope_type=2, riemann="hllc", pool_octs=1 << 20, device=0, tile=None):
        self.L = lib()
        check(self.L.rh_init(device), "rh_init")
        self.precision = PRECISION[precision] if isinstance(precision, str) else int(precision)
        r = RH_RIEMANN[riemann] if isinstance(riemann, str) else int(riemann)
        check(self.L.rh_batch_init(self.precision, int(slope_type), r, int(pool_octs)), "rh_batch_init")
        self.problems = {}
        if tile is not None:
            self.set_tile(*tile)

    def footprint(self, p):
        return int(self.L.rh_batch_footprint(C.byref(p)))

    def add(self, p, ic):
        """Problem id, or None when the pool has no room (RH_ENOMEM)."""
        i = C.c_int()
        rc = self.L.rh_batch_add(C.byref(p), C.byref(ic), C.byref(i))
        if rc == RH_ENOMEM:
            return None
        check(rc, "rh_batch_add")
        self.problems[i.value] = (tuple(p.n), p)
        return i.value

    def remove(self, pid):
        check(self.L.rh_batch_remove(int(pid)), "rh_batch_remove")
        self.problems.pop(pid, None)

    def step(self, nsteps=1):
        check(self.L.rh_batch_step(int(nsteps)), "rh_batch_step")

    def status(self, pid):
        t, dt = C.c_double(), C.c_double()
        ns, done = C.c_int(), C.c_int()
        tot = (C.c_double * 5)()
        check(self.L.rh_batch_status(int(pid), C.byref(t), C.byref(ns), C.byref(done), C.byref(dt), tot),
              "rh_batch_status")
        return {"t": t.value, "nstep": ns.value, "done": bool(done.value), "dt": dt.value, "totals": list(tot)}

    def poll(self):
        """(done, nstep, t) arrays over all problem slots."""
        cap = self.L.rh_batch_capacity()
        done = np.zeros(cap, np.int32)
        ns = np.zeros(cap, np.int32)
        t = np.zeros(cap, np.float64)
        check(self.L.rh_batch_poll(done.ctypes.data_as(C.POINTER(C.c_int)), ns.ctypes.data_as(C.POINTER(C.c_int)),
                                   dptr(t)), "rh_batch_poll")
        return done, ns, t

    def fetch(self, pid):
        n, _ = self.problems[pid]
        out = np.empty(((n[0] // 2) * (n[1] // 2) * (n[2] // 2), 5, 8))
        check(self.L.rh_batch_fetch(int(pid), dptr(out)), "rh_batch_fetch")
        return out

    def fetch_dense(self, pid):
        return octs_to_dense(self.fetch(pid), self.problems[pid][0])

    def file_image(self, pid, kind):
        """Bytes of a problem's amr / hydro_backup / hydro_output file (one
        level 1 of n/2 octs per axis, row-major octs)."""
        from .files import batch_image
        return batch_image(pid, kind)

    def write_output(self, pid, root, number, backup=False):
        """output_NNNNN (or backup_NNNNN) directory of one problem under root;
        returns its path.  The cell size dx is boxlen/2 (level 1)."""
        from . import files
        n, p = self.problems[pid]
        st = self.status(pid)
        noct = (n[0] // 2) * (n[1] // 2) * (n[2] // 2)
        path = files.dir_name(root, number, backup)
        info = files.info_txt(1, 1, noct, st["nstep"], 2.0 * p.dx, st["t"], p.gamma)
        files.write_dir(path, self.file_image(pid, "amr"),
                        self.file_image(pid, "hydro_backup" if backup else "hydro_output"), info, backup)
        return path

    def set_tile(self, txo, tyo, minb, lz):
        check(self.L.rh_batch_set_tile(int(txo), int(tyo), int(minb), int(lz)), "rh_batch_set_tile")

    def tiles(self):
        """Compiled (txo, tyo, minb) shapes of the batch kernel at this precision."""
        tx, ty, mb = (C.c_int * 64)(), (C.c_int * 64)(), (C.c_int * 64)()
        n = self.L.rh_batch_list_tiles(self.precision, tx, ty, mb, 64)
        return [(tx[i], ty[i], mb[i]) for i in range(min(n, 64))]

    def tune(self, lz_choices=(8, 16, 32), nsteps=2, reps=3, log=None):
        """Autotune the batch kernel on the problems currently in the batch:
        time every compiled (txo, tyo, minb) x lz with CUDA events (median of
        ``reps`` runs of ``nsteps`` steps; the problems advance meanwhile, so
        give them a stopping rule far away), keep the fastest selected and
        return (best, table)."""
        table = []
        for (tx, ty, mb) in self.tiles():
            for lz in lz_choices:
                self.set_tile(tx, ty, mb, lz)
                self.bench(1)  # rebuilds the work list and the step graph
                ms = float(np.median([self.bench(nsteps) for _ in range(reps)]))
                table.append({"txo": tx, "tyo": ty, "minb": mb, "lz": lz, "ms": ms})
                if log:
                    log("batch autotune %dx%d minb=%d lz=%d: %.3f ms/step" % (tx, ty, mb, lz, ms))
        best = min(table, key=lambda r: r["ms"])
        self.set_tile(best["txo"], best["tyo"], best["minb"], best["lz"])
        return best, table

    def bench(self, nsteps):
        ms = C.c_float()
        check(self.L.rh_batch_bench(int(nsteps), C.byref(ms)), "rh_batch_bench")
        return ms.value

    def set_state_check(self, on=True):
        """Check every stepped problem after each step; a problem with a NaN/Inf,
        rho <= 0 or internal energy <= 0 cell stops with done == 2."""
        check(self.L.rh_batch_set_state_check(int(bool(on))), "rh_batch_set_state_check")

    def check_mask(self, pid):
        """The state check's bits of a problem (0: clean)."""
        m = C.c_int()
        check(self.L.rh_batch_check_mask(int(pid), C.byref(m)), "rh_batch_check_mask")
        return m.value

    def cells(self):
        """Cells one step updates (unfinished problems)."""
        return int(self.L.rh_batch_cells())

    def close(self):
        check(self.L.rh_batch_free(), "rh_batch_free")


def random_state(rng, gamma):
    """Primitive (rho, u, v, w, p): rho log-uniform in [1e-3, 1e3], p
    log-uniform in [1e-4, 1e2], |v| uniform in [0, 3] sound speeds, random direction."""
    rho = 10 ** rng.uniform(-3, 3)
    p = 10 ** rng.uniform(-4, 2)
    cs = np.sqrt(gamma * p / rho)
    d = rng.standard_normal(3)
    d *= rng.uniform(0, 3) * cs / np.linalg.norm(d)
    return [rho, d[0], d[1], d[2], p]


def riemann_blast_ensemble(n_problems=1024, seed=20261203, sides=(16, 32, 48, 64, 96, 128), steps=50,
                           blast_fraction=0.25):
    """Independent 3D Riemann and blast problems of uneven size: cubic boxes
    with sides drawn uniformly from ``sides`` (unit box, outflow), gamma
    uniform in [1.1, 1.67]; a Riemann problem splits two random states along a
    random axis, a blast puts a pressure 100x above the larger of the two
    inside a sphere of radius 0.05-0.15 around a random centre.  Returns a list
    of (rh_batch_problem, rh_batch_ic)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_problems):
        s = int(rng.choice(sides))
        g = float(rng.uniform(1.1, 1.67))
        a, b = random_state(rng, g), random_state(rng, g)
        p = problem((s, s, s), dx=1.0 / s, bc="outflow", gamma=g, courant_factor=0.8, max_steps=steps)
        if rng.uniform() < blast_fraction:
            ic = ic_blast(a, 100.0 * max(a[4], b[4]), rng.uniform(0.05, 0.15), rng.uniform(0.3, 0.7, 3))
        else:
            ic = ic_split(int(rng.integers(0, 3)), a, b)
        out.append((p, ic))
    return out


def ensemble_octs(ensemble):
    return sum((p.n[0] // 2) * (p.n[1] // 2) * (p.n[2] // 2) for p, _ in ensemble)
