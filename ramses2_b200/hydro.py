"""Host-side mirror of the reference's hydro leaf calls, backed by librh_b200.so.

:class:`GodunovGPU` exposes the per-level calls a RAMSES II host makes in one
coarse step (amr/amr_step.f90:276-455) with the reference's names and argument
meaning: ``courant_fine`` (r_courant_fine, hydro/courant_fine.f90:18-52),
``set_unew`` / ``set_uold`` (hydro/godunov_fine.f90:84-214) and
``godunov_fine`` (hydro/godunov_fine.f90:13-79).  Each call goes through the C
ABI (include/ramses_hydro.h) exactly as the Fortran shim would.
"""
import ctypes as C
import os

import numpy as np

from ._abi import RH_PREC_FP32_BULK, RH_PREC_FP64, dptr
from ._lib import check, lib

PRECISION = {"fp64": RH_PREC_FP64, "fp32_bulk": RH_PREC_FP32_BULK, "fp32": RH_PREC_FP32_BULK}


class GodunovGPU:
    """One mesh resident on one B200, stepped through the C ABI."""

    def __init__(self, mesh, params, precision="fp64", device=0, tile=None, amr_tile=None, table_builder=None,
                 deterministic=False):
        self.mesh = mesh
        self.params = params
        self.L = lib()
        check(self.L.rh_init(device), "rh_init")
        self.precision = PRECISION[precision] if isinstance(precision, str) else int(precision)
        check(self.L.rh_set_precision(self.precision), "rh_set_precision")
        if tile is not None:
            self.set_tile(*tile)
        check(self.L.rh_set_interpolation(params.interpol_var, params.interpol_type), "rh_set_interpolation")
        if amr_tile is not None:
            check(self.L.rh_set_amr_tile(*amr_tile), "rh_set_amr_tile")
        if table_builder is not None:
            check(self.L.rh_set_table_builder({"host": 0, "device": 1}.get(table_builder, table_builder)),
                  "rh_set_table_builder")
        check(self.L.rh_set_deterministic(int(bool(deterministic))), "rh_set_deterministic")
        self._desc = mesh.desc()
        check(self.L.rh_set_mesh(C.byref(self._desc), dptr(mesh.uold), 5, 8), "rh_set_mesh")
        g = np.ascontiguousarray(mesh.gravity, np.float64)
        self._grav = g

    # ---- reference leaf calls -------------------------------------------------
    def courant_fine(self, ilevel):
        """(mass, ekin, eint, emag, dt) of the leaf cells of a level."""
        m = self.mesh
        out = [C.c_double() for _ in range(5)]
        P = self.params
        check(self.L.rh_cmpdt(int(m.head[ilevel]), int(m.noct[ilevel]), m.dx(ilevel), P.gamma, P.smallr,
                              P.smallc, P.courant_factor, dptr(self._grav), *[C.byref(o) for o in out]),
              "rh_cmpdt")
        return np.array([o.value for o in out])

    def set_unew(self, ilevel):
        m = self.mesh
        check(self.L.rh_set_unew(int(m.head[ilevel]), int(m.noct[ilevel])), "rh_set_unew")

    def set_uold(self, ilevel):
        m = self.mesh
        check(self.L.rh_set_uold(int(m.head[ilevel]), int(m.noct[ilevel])), "rh_set_uold")

    def godunov_fine(self, ilevel, dt):
        m = self.mesh
        P = self.params
        n3 = m.nsubgrid ** 3
        head_sub = (int(m.head[ilevel]) - 1) // n3 + 1
        nsub = int(m.noct[ilevel]) // n3
        dx = m.dx(ilevel)
        smax_cap = P.courant_factor * dx / dt
        check(self.L.rh_godunov(head_sub, nsub, m.ngridmax, ilevel, m.levelmin, m.levelmax, P.gamma, P.smallr,
                                P.smallc ** 2, dt, dx, smax_cap, P.slope_type, P.riemann, dptr(self._grav)),
              "rh_godunov")

    def upload_fine(self, ilevel):
        """Restriction of level ilevel+1 into the refined cells of level ilevel."""
        m = self.mesh
        P = self.params
        if ilevel >= m.levelmax or not m.noct[ilevel + 1]:
            return
        check(self.L.rh_upload(int(m.head[ilevel + 1]), int(m.noct[ilevel + 1]), int(P.interpol_var == 1),
                               P.gamma, P.smallr, P.smallc ** 2), "rh_upload")

    def hydro_flag(self, ilevel, flags, flag1):
        """Gradient refinement flags of level ilevel (hydro_flag): flag1 is the
        (ngridmax, 8) int32 array of the host; returns the newly flagged count."""
        assert flag1.dtype == np.int32 and flag1.flags.c_contiguous and flag1.size == 8 * self.mesh.ngridmax
        n = C.c_longlong()
        P = self.params
        check(self.L.rh_hydro_flag(int(ilevel), C.byref(flags), P.gamma, P.smallr,
                                   flag1.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n)), "rh_hydro_flag")
        return n.value

    def check_state(self, ilevel):
        """The reference's debug scan of a level's uold (gpu_check_nan):
        (bad cells, first bad oct 1-based or 0, mask: 1 NaN/Inf, 2 rho<=0,
        4 internal energy<=0)."""
        m = self.mesh
        nbad, first, mask = C.c_int(), C.c_int(), C.c_int()
        check(self.L.rh_check_state(int(m.head[ilevel]), int(m.noct[ilevel]), C.byref(nbad), C.byref(first),
                                    C.byref(mask)), "rh_check_state")
        return nbad.value, first.value, mask.value

    def set_state_check(self, on=True):
        """Make coarse_step check every level after the step (RH_EBADSTATE)."""
        check(self.L.rh_set_state_check(int(bool(on))), "rh_set_state_check")

    # ---- conveniences -----------------------------------------------------------
    def step_uniform(self, dt=None):
        """One coarse step of a single-level run in the reference's order."""
        lev = self.mesh.levelmin
        out = self.courant_fine(lev)
        dtnew = min(self.mesh.dx(lev) / self.params.smallc, out[4]) if dt is None else dt
        self.set_unew(lev)
        self.godunov_fine(lev, dtnew)
        self.set_uold(lev)
        return dtnew, out

    def fetch_uold(self):
        """Device uold copied back in the reference layout (N, 5, 8)."""
        u = np.empty_like(self.mesh.uold)
        check(self.L.rh_transfer_grid_host(dptr(u), self.mesh.ngridmax, 5, 8), "rh_transfer_grid_host")
        return u

    def push_uold(self, u=None):
        u = self.mesh.uold if u is None else np.ascontiguousarray(u, np.float64)
        check(self.L.rh_set_grid_device(dptr(u), self.mesh.ngridmax, 5, 8), "rh_set_grid_device")

    def sync(self):
        check(self.L.rh_sync(), "rh_sync")

    def coarse_step(self, dt=None):
        """amr_coarse_step in one library call (rh_coarse_step): returns dt."""
        d = C.c_double(0.0 if dt is None else float(dt))
        check(self.L.rh_coarse_step(C.byref(self.params), C.byref(d), None), "rh_coarse_step")
        return d.value

    def coarse_step_host(self, host_in, host_out=None, dt=None):
        """rh_coarse_step_host: one coarse step of a state held on the host
        (host_in, the reference layout; written to host_out, default host_in),
        the copies overlapped with the pencils.  Returns (dt taken, dt_next)."""
        host_out = host_in if host_out is None else host_out
        for a in (host_in, host_out):
            assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape == self.mesh.uold.shape
        d = C.c_double(0.0 if dt is None else float(dt))
        nxt = C.c_double()
        check(self.L.rh_coarse_step_host(C.byref(self.params), C.c_void_p(host_in.ctypes.data),
                                         C.c_void_p(host_out.ctypes.data), C.byref(d), C.byref(nxt)),
              "rh_coarse_step_host")
        return d.value, nxt.value

    # ---- restart / snapshot files (include/ramses_hydro_io.h) -------------------
    def file_image(self, kind):
        """Bytes of the amr / hydro_backup / hydro_output file of the current state."""
        from .files import context_image
        return context_image(kind, self.params.gamma)

    def write_output(self, root, number, time=0.0, nstep_coarse=0, backup=False):
        """output_NNNNN (or backup_NNNNN) directory of the current state under
        root, in the reference's layout; returns its path."""
        from . import files
        m = self.mesh
        path = files.dir_name(root, number, backup)
        info = files.info_txt(m.levelmin, m.levelmax, m.ngridmax, nstep_coarse, m.boxlen, time, self.params.gamma)
        files.write_dir(path, self.file_image("amr"), self.file_image("hydro_backup" if backup else "hydro_output"),
                        info, backup)
        return path

    def restore(self, hydro_backup):
        """Restart: uold from a hydro backup image (bytes) or a backup directory."""
        from . import files
        if isinstance(hydro_backup, str):
            with open(os.path.join(hydro_backup, "hydro.00001"), "rb") as f:
                hydro_backup = f.read()
        files.restore_hydro(hydro_backup)

    def set_tile(self, txo, tyo, lz, minb=None):
        """Pencil tile (txo x tyo octs, lz layers); minb defaults to the
        compiled variant with the most CTAs per SM for this shape."""
        if minb is None:
            opts = [b for (x, y, b) in self.tiles() if (x, y) == (txo, tyo)]
            if not opts:
                raise ValueError("tile %dx%d not compiled" % (txo, tyo))
            minb = max(opts)
        check(self.L.rh_set_tile(txo, tyo, minb, lz), "rh_set_tile")

    def tiles(self):
        """Compiled (txo, tyo, minb) shapes of this precision."""
        tx, ty, mb = (C.c_int * 64)(), (C.c_int * 64)(), (C.c_int * 64)()
        n = self.L.rh_list_tiles(self.precision, tx, ty, mb, 64)
        return [(tx[i], ty[i], mb[i]) for i in range(min(n, 64))]

    def bench_godunov(self, ilevel, nrep, dt):
        P = self.params
        ms = C.c_float()
        check(self.L.rh_bench_godunov(ilevel, nrep, P.gamma, P.smallr, P.smallc, dt, self.mesh.dx(ilevel),
                                      P.courant_factor, P.slope_type, P.riemann, C.byref(ms)),
              "rh_bench_godunov")
        return ms.value

    def close(self):
        check(self.L.rh_finalize(), "rh_finalize")


def amr_coarse_step(solver, mesh, dt=None):
    """One coarse step of every level with nsubcycle = 1, in amr/amr_step.f90's
    order: courant_fine of every level (the smallest dt wins,
    amr/amr_step.f90:588), set_unew coarse to fine, then godunov_fine and
    set_uold from the finest level to the coarsest (the coarse update of level
    l lands in unew of level l-1 before that level is stepped).  ``solver`` is
    a :class:`GodunovGPU` (or anything with the same four leaf calls)."""
    lev = [l for l in range(mesh.levelmin, mesh.levelmax + 1) if mesh.noct[l]]
    if dt is None:
        dt = min(min(mesh.dx(l) / solver.params.smallc, solver.courant_fine(l)[4]) for l in lev)
    for l in lev:
        solver.set_unew(l)
    for l in reversed(lev):
        solver.godunov_fine(l, dt)
        solver.set_uold(l)
        if l < lev[-1]:
            solver.upload_fine(l)
    return dt

