"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU checker (librh_oracle.so).

The checker restates RAMSES II's FP64 CPU hydro step (hydro/umuscl.f90,
hydro/godunov_utils.f90, hydro/godunov_fine.f90, hydro/courant_fine.f90).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
Parity status: the Fortran reference binary cannot be built (no Fortran
compiler in the image) and ships no golden vectors for this path; the checker
is pinned against the reference's own code (its Metal hydro and flag shaders
compiled as C++, tests/test_oracle_pin_ref.py; its Python output reader,
tests/test_files_host.py) and by known-answer tests.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from ramses2_b200._abi import FlagParams, HydroParams, MeshDesc, dptr

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librh_oracle.so")
_lib = None


def build():
    """Compile librh_oracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def reference_root():
    """The reference checkout the CPU checks may read (environment variable
    REF_ROOT, else the default of oracle/Makefile), or None when it is absent
    (as on a machine that only runs the tests)."""
    root = os.environ.get("REF_ROOT")
    if not root:
        r = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-ref-root"],
                           capture_output=True, text=True)
        root = r.stdout.strip() if r.returncode == 0 else ""
    return root if root and os.path.isdir(root) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.rh_oracle_riemann.argtypes = [C.c_int, P(C.c_double), P(C.c_double), P(HydroParams),
                                        C.c_double, P(C.c_double)]
        L.rh_oracle_unsplit.argtypes = [C.c_int, P(C.c_double), C.c_double, C.c_double,
                                        P(HydroParams), P(C.c_double)]
        L.rh_oracle_cmpdt.argtypes = [P(C.c_double), P(C.c_double), C.c_double, P(HydroParams), C.c_int]
        L.rh_oracle_cmpdt.restype = C.c_double
        L.rh_oracle_cmpdt_octs.argtypes = [P(C.c_double), C.c_longlong, P(C.c_double), C.c_double, P(HydroParams),
                                           C.c_int, C.c_int]
        L.rh_oracle_cmpdt_octs.restype = C.c_double
        L.rh_oracle_interpol_hydro.argtypes = [P(C.c_double), P(C.c_double), C.c_int, C.c_int, C.c_double]
        L.rh_oracle_godunov_fine.argtypes = [P(MeshDesc), P(HydroParams), C.c_int, C.c_double,
                                             P(C.c_double), P(C.c_double), C.c_int]
        L.rh_oracle_upload_fine.argtypes = [P(MeshDesc), P(HydroParams), C.c_int, P(C.c_double)]
        L.rh_oracle_hydro_flag.argtypes = [P(MeshDesc), P(HydroParams), P(FlagParams), C.c_int, P(C.c_double),
                                           P(C.c_int32), P(C.c_longlong)]
        L.rh_oracle_courant_fine.argtypes = [P(MeshDesc), P(HydroParams), C.c_int, P(C.c_double),
                                             P(C.c_double)]
        L.rh_oracle_output_prims.argtypes = [P(C.c_double), C.c_longlong, C.c_double, P(C.c_float)]
        L.rh_oracle_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle error %d: %s" % (rc, lib().rh_oracle_last_error().decode()))


def riemann(solver, ql, qr, params, smax_cap=np.finfo(np.float64).max):
    ql = np.ascontiguousarray(ql, np.float64)
    qr = np.ascontiguousarray(qr, np.float64)
    out = np.zeros(6)
    _check(lib().rh_oracle_riemann(solver, dptr(ql), dptr(qr), C.byref(params), smax_cap, dptr(out)))
    return out


def unsplit(uin, dx, dt, params):
    """uin: (5, nn+4, nn+4, nn+4) indexed [var, k, j, i] -> flux (3, 5, nn+1, nn+1, nn+1)."""
    nn = uin.shape[-1] - 4
    u = np.ascontiguousarray(uin, np.float64)
    out = np.zeros((3, 5, nn + 1, nn + 1, nn + 1))
    _check(lib().rh_oracle_unsplit(nn, dptr(u), dx, dt, C.byref(params), dptr(out)))
    return out


def cmpdt(uu, dx, params, grav=(0.0, 0.0, 0.0), ndim=3):
    uu = np.ascontiguousarray(uu, np.float64)
    g = np.ascontiguousarray(grav, np.float64)
    return lib().rh_oracle_cmpdt(dptr(uu), dptr(g), dx, C.byref(params), ndim)


def cmpdt_octs(uold, dx, params, ndim=3, grav=(0.0, 0.0, 0.0), nthreads=1):
    """Smallest cell dt (cmpdt) over a (noct, 5, 8) state, in ndim directions."""
    u = np.ascontiguousarray(uold, np.float64)
    g = np.ascontiguousarray(grav, np.float64)
    return lib().rh_oracle_cmpdt_octs(dptr(u), len(u), dptr(g), dx, C.byref(params), ndim, nthreads)


def solve_box(dense, dx, params, bc="outflow", ndim=3, t_end=0.0, max_steps=0, nthreads=1):
    """One single-level problem of the batch runtime solved by the oracle to
    its stopping rule, in the order the batch follows (the reference's coarse
    step, amr/amr_step.f90, with newdt_fine's dt = min(dx/smallc, courant
    dt) cut to land on t_end): courant_fine dt of the state (ndim
    directions; a 2D problem is a two-cell-deep periodic z slab), set_unew,
    godunov_fine, set_uold, until t >= t_end (relative 1e-12) or max_steps
    steps.  dense: (5, nz, ny, nx) conserved state of even extents.
    Returns (final dense state, t, steps)."""
    from ramses2_b200.mesh import uniform_mesh

    nz, ny, nx = dense.shape[1:]
    m = uniform_mesh(1, nsubgrid=1, boxlen=2.0 * dx, bc=bc, box_nx=(nx // 2, ny // 2, nz // 2))
    assert m.dx(1) == dx
    m.from_dense(dense, 1)
    o = OracleHydro(m, params, nthreads=nthreads)
    t, ns = 0.0, 0
    while True:
        dt = min(dx / params.smallc, cmpdt_octs(m.uold, dx, params, ndim=ndim, nthreads=nthreads))
        if t_end > 0.0 and t + dt > t_end:
            dt = t_end - t
        o.step_uniform(dt)
        t += dt
        ns += 1
        if (t_end > 0.0 and t >= t_end * (1.0 - 1e-12)) or (max_steps > 0 and ns >= max_steps):
            return m.to_dense(m.uold, 1), t, ns


def interpol_hydro(u1, interpol_var, interpol_type, smallr=1e-10):
    """u1: (5, 7) [var, j] -> u2 (5, 8) [var, ind]."""
    a = np.ascontiguousarray(u1, np.float64)
    out = np.zeros((5, 8))
    _check(lib().rh_oracle_interpol_hydro(dptr(a), dptr(out), interpol_var, interpol_type, smallr))
    return out


def output_prims(uold, gamma):
    """output_hydro's float32 primitives (hydro/output_hydro.f90:86-140) of
    uold (noct, 5, 8) -> (noct, 5, 8) float32 = (rho, u, v, w, p)."""
    u = np.ascontiguousarray(uold, np.float64)
    q = np.zeros(u.shape, np.float32)
    _check(lib().rh_oracle_output_prims(dptr(u), u.shape[0], float(gamma), q.ctypes.data_as(C.POINTER(C.c_float))))
    return q


FILE_AMR, FILE_HYDRO_BACKUP, FILE_HYDRO_OUTPUT = 1, 2, 3


def file_image(kind, uold, grid, head, noct, levelmin, levelmax, gamma=None):
    """Bytes of one rank's amr or hydro file, restated from the writers:

    * header: int32 ndim, [nvar,] levelmin, nlevelmax, noct(levelmin:nlevelmax)
      (amr/output_amr.f90:702-707 backup_amr; hydro/output_hydro.f90:208-218
      backup_hydro; amr/ramses_commons.f90:138-158 open_file);
    * amr: per level, per oct (head(l) .. tail(l)): int32 ckey(1:3) and the
      refined bits, bit ind-1 set for a refined cell (output_amr.f90:712-727);
    * hydro backup: per oct float64 uold(1:8,1:5) (output_hydro.f90:223-237);
    * hydro output: per oct float32 q(1:8,1:5) of output_prims
      (output_hydro.f90:77-149).

    uold (ngridmax, 5, 8); grid OCT_DTYPE records; head/noct indexed by level.
    """
    levels = range(levelmin, levelmax + 1)
    hdr = [3] + ([] if kind == FILE_AMR else [5]) + [levelmin, levelmax] + [int(noct[l]) for l in levels]
    parts = [np.asarray(hdr, "<i4").tobytes()]
    for l in levels:
        a, n = int(head[l]) - 1, int(noct[l])
        if n == 0:
            continue
        if kind == FILE_AMR:
            g = grid[a:a + n]
            rec = np.zeros((n, 4), "<i4")
            rec[:, :3] = g["ckey"]
            rec[:, 3] = ((g["refined"] != 0).astype(np.int64) << np.arange(8)).sum(axis=1)
            parts.append(rec.tobytes())
        elif kind == FILE_HYDRO_BACKUP:
            parts.append(np.ascontiguousarray(uold[a:a + n], "<f8").tobytes())
        elif kind == FILE_HYDRO_OUTPUT:
            parts.append(output_prims(uold[a:a + n], gamma).astype("<f4").tobytes())
        else:
            raise ValueError("unknown file kind %r" % (kind,))
    return b"".join(parts)


def restart_offsets(kind, levelmin, levelmax, noct):
    """0-based byte offset of each level's first oct in a backup file, from
    the restart reader's formulas (amr/init_refine_restart.f90:387,396, 1-based):
    13 + 4*nlevel + 16*nskip (amr), 17 + 4*nlevel + 320*nskip (hydro)."""
    nlev = levelmax - levelmin + 1
    base, rec = (13, 16) if kind == FILE_AMR else (17, 8 * 8 * 5)
    off, nskip = {}, 0
    for l in range(levelmin, levelmax + 1):
        off[l] = base + 4 * nlev + rec * nskip - 1
        nskip += int(noct[l])
    return off


class OracleHydro:
    """The reference's per-level leaf calls, restated on the CPU.

    Mirrors r_courant_fine / r_set_unew / r_godunov_fine / r_set_uold
    (hydro/courant_fine.f90:18-52, hydro/godunov_fine.f90:13-214) on a
    :class:`ramses2_b200.mesh.Mesh`.
    """

    def __init__(self, mesh, params, nthreads=1):
        self.mesh = mesh
        self.params = params
        self.nthreads = nthreads
        self.unew = mesh.uold.copy()

    def courant_fine(self, ilevel):
        out = np.zeros(5)
        _check(lib().rh_oracle_courant_fine(C.byref(self.mesh.desc()), C.byref(self.params), ilevel,
                                            dptr(self.mesh.uold), dptr(out)))
        return out  # mass, ekin, eint, emag, dt

    def set_unew(self, ilevel):
        sl = self.mesh.level_slice(ilevel)
        self.unew[sl] = self.mesh.uold[sl]

    def set_uold(self, ilevel):
        sl = self.mesh.level_slice(ilevel)
        self.mesh.uold[sl] = self.unew[sl]

    def godunov_fine(self, ilevel, dt):
        _check(lib().rh_oracle_godunov_fine(C.byref(self.mesh.desc()), C.byref(self.params), ilevel,
                                            dt, dptr(self.mesh.uold), dptr(self.unew), self.nthreads))

    def upload_fine(self, ilevel):
        """Restriction of level ilevel+1 into level ilevel (hydro/upload.f90:74-271)."""
        _check(lib().rh_oracle_upload_fine(C.byref(self.mesh.desc()), C.byref(self.params), ilevel,
                                           dptr(self.mesh.uold)))

    def hydro_flag(self, ilevel, flags, flag1):
        """Gradient branch of hydro_flag (hydro/hydro_flag.f90:7-159) on the
        (ngridmax, 8) int32 flag1; returns the newly flagged count."""
        n = C.c_longlong()
        _check(lib().rh_oracle_hydro_flag(C.byref(self.mesh.desc()), C.byref(self.params), C.byref(flags), ilevel,
                                          dptr(self.mesh.uold), flag1.ctypes.data_as(C.POINTER(C.c_int32)),
                                          C.byref(n)))
        return n.value

    def step_uniform(self, dt=None):
        """One coarse step of a single-level run (amr/amr_step.f90:276-455 order)."""
        lev = self.mesh.levelmin
        out = self.courant_fine(lev)
        dx = self.mesh.dx(lev)
        dtnew = min(dx / self.params.smallc, out[4]) if dt is None else dt
        self.set_unew(lev)
        self.godunov_fine(lev, dtnew)
        self.set_uold(lev)
        return dtnew, out
