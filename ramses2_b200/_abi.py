"""ctypes mirrors of the C ABI types declared in include/ramses_hydro.h.

``OCT_DTYPE`` is the numpy view of ``type(oct)`` (amr/oct_commons.f90:5-10,
NDIM=3, nhilbert=1): 32-byte records, so a Fortran ``grid(1:ngridmax)`` array
and a numpy array of this dtype share one memory layout.
"""
import ctypes as C

import numpy as np

OCT_DTYPE = np.dtype(
    [("hkey", "<i8"), ("ckey", "<i4", (3,)), ("refined", "u1", (8,)), ("lev", "<i4")],
    align=False,
)
assert OCT_DTYPE.itemsize == 32

RH_RIEMANN = {"llf": 1, "hll": 2, "hllc": 3}
RH_BOUND_PERIODIC = 0
RH_BOUND_REFLEXIVE = 1
RH_BOUND_ZERO_GRADIENT = 2
RH_PREC_FP64 = 0
RH_PREC_FP32_BULK = 1

STATUS = {
    0: "RH_OK",
    1: "RH_EINVAL",
    2: "RH_ENOMEM",
    3: "RH_ECUDA",
    4: "RH_ESTATE",
    5: "RH_ETIMEDOUT",
    6: "RH_ENODEV",
    7: "RH_EBUSY",
    8: "RH_EBADSTATE",
}


class HydroParams(C.Structure):
    """hydro_params_t subset (amr/amr_commons.f90:690-702)."""

    _fields_ = [
        ("gamma", C.c_double),
        ("smallr", C.c_double),
        ("smallc", C.c_double),
        ("courant_factor", C.c_double),
        ("difmag", C.c_double),
        ("slope_type", C.c_int32),
        ("riemann", C.c_int32),
        ("interpol_var", C.c_int32),
        ("interpol_type", C.c_int32),
    ]

    @classmethod
    def make(cls, gamma=1.4, smallr=1e-10, smallc=1e-10, courant_factor=0.8,
             slope_type=2, riemann="hllc", interpol_var=0, interpol_type=0, difmag=0.0):
        r = RH_RIEMANN[riemann] if isinstance(riemann, str) else int(riemann)
        return cls(gamma, smallr, smallc, courant_factor, difmag, slope_type, r,
                   interpol_var, interpol_type)


class MeshDesc(C.Structure):
    """rh_mesh_desc: the reference's flat-oct mesh (amr/amr_commons.f90 mesh_t)."""

    _fields_ = [
        ("nsubgrid", C.c_int32),
        ("levelmin", C.c_int32),
        ("levelmax", C.c_int32),
        ("ngridmax", C.c_int32),
        ("box_nx", C.c_int32 * 3),
        ("periodic", C.c_int32 * 3),
        ("bound_type", C.c_int32 * 6),
        ("boxlen", C.c_double),
        ("constant_gravity", C.c_double * 3),
        ("head", C.POINTER(C.c_int32)),
        ("noct", C.POINTER(C.c_int32)),
        ("grid", C.c_void_p),
    ]


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array."""
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


RH_IC_SPLIT = 1
RH_IC_BLAST = 2
RH_IC_HOST = 3


class BatchProblem(C.Structure):
    """rh_batch_problem (include/ramses_hydro_batch.h)."""

    _fields_ = [
        ("n", C.c_int32 * 3),
        ("ndim", C.c_int32),
        ("bound_type", C.c_int32 * 6),
        ("dx", C.c_double),
        ("gamma", C.c_double),
        ("smallr", C.c_double),
        ("smallc", C.c_double),
        ("courant_factor", C.c_double),
        ("t_end", C.c_double),
        ("max_steps", C.c_int32),
    ]


class BatchIC(C.Structure):
    """rh_batch_ic (include/ramses_hydro_batch.h)."""

    _fields_ = [
        ("kind", C.c_int32),
        ("axis", C.c_int32),
        ("left", C.c_double * 5),
        ("right", C.c_double * 5),
        ("ambient", C.c_double * 5),
        ("p_in", C.c_double),
        ("radius", C.c_double),
        ("centre", C.c_double * 3),
        ("host_uold", C.c_void_p),
    ]


class FlagParams(C.Structure):
    """rh_flag_params: hydro_refine's gradient criteria (negative = off)."""

    _fields_ = [("err_grad_d", C.c_double), ("err_grad_p", C.c_double), ("err_grad_u", C.c_double),
                ("floor_d", C.c_double), ("floor_p", C.c_double), ("floor_u", C.c_double)]

    @classmethod
    def make(cls, err_grad_d=-1.0, err_grad_p=-1.0, err_grad_u=-1.0, floor_d=1e-10, floor_p=1e-10, floor_u=1e-10):
        return cls(err_grad_d, err_grad_p, err_grad_u, floor_d, floor_p, floor_u)
