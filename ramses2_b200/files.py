"""Restart (backup) and snapshot (output) directories of the hydro state in
the reference's layouts, from the device-resident state.

The binary files come from the library (include/ramses_hydro_io.h:
``rh_file_image`` / ``rh_batch_file_image``), assembled on the device; this
module adds the text files of an output directory and names everything as the
reference's dump does for one rank (amr/output_amr.f90:56-230 dump_all):

    output_NNNNN/  info.txt  hydro_header.txt  amr.00001  hydro.00001
    backup_NNNNN/  info.txt  hydro_header.txt  amr.00001  hydro.00001

``info.txt`` follows output_info (amr/output_amr.f90:740-791) and
``hydro_header.txt`` file_descriptor_hydro (hydro/output_hydro.f90:251-385),
hydro variables only.  The reference's other backup files (params.bin,
namelist.txt, particles, gravity) belong to parts of the code outside the hydro
step and are not written.
"""
import ctypes as C
import os

import numpy as np

from ._lib import check, lib

FILE_AMR, FILE_HYDRO_BACKUP, FILE_HYDRO_OUTPUT = 1, 2, 3
KINDS = {"amr": FILE_AMR, "hydro_backup": FILE_HYDRO_BACKUP, "hydro_output": FILE_HYDRO_OUTPUT}


def fortran_e(x, d=15, w=23):
    """Fortran ``Ew.d`` edit of a real: 0.ddd...E+xx right-justified in w."""
    x = float(x)
    if x == 0.0 or not np.isfinite(x):
        body = ("0." + "0" * d + "E+00") if x == 0.0 else str(x).upper()
        if x == 0.0 and np.signbit(x):
            body = "-" + body
        return body.rjust(w)
    s = "%.*e" % (d - 1, abs(x))
    mant, ex = s.split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    es = "E%+03d" % e if abs(e) < 100 else "%+04d" % e
    body = ("-" if x < 0 else "") + "0." + digits + es
    return body.rjust(w)


def info_txt(levelmin, levelmax, ngridmax, nstep_coarse=0, boxlen=1.0, time=0.0, gamma=1.4, ndim=3, nfile=1,
             ncpu=1, texp=0.0, aexp=1.0, h0=1.0, omega_m=1.0, omega_l=0.0, omega_k=0.0, omega_b=0.0,
             unit_l=1.0, unit_d=1.0, unit_t=1.0):
    """info.txt as output_info writes it (amr/output_amr.f90:764-786)."""
    ints = [("nfile", nfile), ("ncpu", ncpu), ("ndim", ndim), ("levelmin", levelmin), ("levelmax", levelmax),
            ("ngridmax", ngridmax), ("nstep_coarse", nstep_coarse)]
    reals = [("boxlen", boxlen), ("time", time), ("texp", texp), ("aexp", aexp), ("H0", h0), ("omega_m", omega_m),
             ("omega_l", omega_l), ("omega_k", omega_k), ("omega_b", omega_b), ("gamma", gamma),
             ("unit_l", unit_l), ("unit_d", unit_d), ("unit_t", unit_t)]
    lines = ["%-12s=%11d" % (k, v) for k, v in ints] + [""]
    lines += ["%-12s=%s" % (k, fortran_e(v)) for k, v in reals] + [""]
    return "\n".join(lines) + "\n"


def hydro_header_txt(backup):
    """hydro_header.txt of file_descriptor_hydro (hydro/output_hydro.f90:271-326)."""
    names = (["density", "momentum_x", "momentum_y", "momentum_z", "total_energy"] if backup else
             ["density", "velocity_x", "velocity_y", "velocity_z", "thermal_pressure"])
    lines = ["nvar        =%11d" % len(names)]
    lines += ["variable #%2d: %s" % (i + 1, n) for i, n in enumerate(names)]
    return "\n".join(lines) + "\n"


def parse_image(image, kind):
    """Header and per-level payload of an amr or hydro file image (bytes).

    Returns dict(ndim, nvar, levelmin, levelmax, noct, levels): levels maps a
    level to (ckey (n, 3) int32, refined bits (n,) int32) for an amr file, to
    (n, nvar, 8) float64 for a backup, float32 for an output."""
    kind = KINDS.get(kind, kind)
    b = bytes(image)
    h = np.frombuffer(b, "<i4", count=4 if len(b) >= 16 else 3)
    if kind == FILE_AMR:
        ndim, nvar, lmin, lmax, hs = int(h[0]), 0, int(h[1]), int(h[2]), 12
    else:
        ndim, nvar, lmin, lmax, hs = int(h[0]), int(h[1]), int(h[2]), int(h[3]), 16
    nlev = lmax - lmin + 1
    if nlev < 1 or hs + 4 * nlev > len(b):
        raise ValueError("file image header is inconsistent")
    noct = np.frombuffer(b, "<i4", count=nlev, offset=hs).astype(np.int64)
    rec = 16 if kind == FILE_AMR else (8 if kind == FILE_HYDRO_BACKUP else 4) * 8 * nvar
    if len(b) != hs + 4 * nlev + rec * int(noct.sum()):
        raise ValueError("file image of %d bytes does not match its header" % len(b))
    off = hs + 4 * nlev
    levels = {}
    for i, l in enumerate(range(lmin, lmax + 1)):
        k = int(noct[i])
        if kind == FILE_AMR:
            r = np.frombuffer(b, "<i4", count=4 * k, offset=off).reshape(k, 4)
            levels[l] = (r[:, :3].copy(), r[:, 3].copy())
        else:
            dt = "<f8" if kind == FILE_HYDRO_BACKUP else "<f4"
            levels[l] = np.frombuffer(b, dt, count=k * nvar * 8, offset=off).reshape(k, nvar, 8).copy()
        off += rec * k
    return dict(ndim=ndim, nvar=nvar, levelmin=lmin, levelmax=lmax,
                noct={l: int(noct[i]) for i, l in enumerate(range(lmin, lmax + 1))}, levels=levels)


def write_dir(path, amr_image, hydro_image, info, backup):
    """One rank's output (or backup) directory from the two file images."""
    os.makedirs(path, exist_ok=True)
    with open(os.path.join(path, "amr.00001"), "wb") as f:
        f.write(amr_image)
    with open(os.path.join(path, "hydro.00001"), "wb") as f:
        f.write(hydro_image)
    with open(os.path.join(path, "hydro_header.txt"), "w") as f:
        f.write(hydro_header_txt(backup))
    with open(os.path.join(path, "info.txt"), "w") as f:
        f.write(info)


def dir_name(root, number, backup=False):
    """output_NNNNN / backup_NNNNN under root (title(): 5 digits)."""
    return os.path.join(root, ("backup_" if backup else "output_") + "%05d" % int(number))


def _image(size_fn, image_fn):
    n = C.c_longlong()
    check(size_fn(C.byref(n)), "file image size")
    buf = np.empty(max(int(n.value), 1), np.uint8)
    got = C.c_longlong()
    check(image_fn(buf.ctypes.data_as(C.c_void_p), int(buf.size), C.byref(got)), "file image")
    return buf[:got.value].tobytes()


def context_image(kind, gamma=1.4):
    """File image (bytes) of the library's current mesh and state."""
    L = lib()
    kind = KINDS.get(kind, kind)
    return _image(lambda n: L.rh_file_size(kind, n),
                  lambda p, cap, got: L.rh_file_image(kind, float(gamma), p, cap, got))


def batch_image(pid, kind):
    """File image (bytes) of one batch problem (a level-1 box of row-major octs)."""
    L = lib()
    kind = KINDS.get(kind, kind)
    n = C.c_longlong()
    L.rh_batch_file_image(int(pid), kind, None, 0, C.byref(n))  # sizes the image
    buf = np.empty(max(int(n.value), 1), np.uint8)
    got = C.c_longlong()
    check(L.rh_batch_file_image(int(pid), kind, buf.ctypes.data_as(C.c_void_p), int(buf.size), C.byref(got)),
          "rh_batch_file_image")
    return buf[:got.value].tobytes()


def restore_hydro(image):
    """Load uold of the library's mesh from a hydro backup image (restart)."""
    b = np.frombuffer(bytes(image), np.uint8)
    check(lib().rh_restore_hydro(b.ctypes.data_as(C.c_void_p), int(b.size)), "rh_restore_hydro")
