"""The allocation-free Courant entry point (rh_cmpdt_noalloc), for callers
that cannot let a library allocate device memory: it must return what the
regular entry point (rh_cmpdt) returns for the same resident state, on two
calls in a row (the second call reuses the shared static scratch), and must
refuse sizes beyond its fixed scratch.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from ramses2_b200._abi import HydroParams
from ramses2_b200._lib import lib
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import riemann3d_state, uniform_mesh

pytestmark = pytest.mark.gpu


def _bind(L):
    f = L.rh_cmpdt_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.POINTER(C.c_double), C.c_void_p, C.c_void_p]
    return f


def test_noalloc_cmpdt_matches_rh_cmpdt_on_two_calls():
    import torch

    L = lib()
    f = _bind(L)
    lev = 5
    m = uniform_mesh(lev, nsubgrid=1, bc="outflow")
    rng = np.random.default_rng(4)
    g, dense = riemann3d_state(rng, 2 * (1 << (lev - 1)), gamma=1.4)
    m.from_dense(dense, lev)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc")
    grav = np.zeros(3)
    gpu = GodunovGPU(m, P, precision="fp64")
    try:
        out = torch.empty(5, dtype=torch.float64, device="cuda")
        dx = m.dx(lev)
        for call in range(2):
            expected = gpu.courant_fine(lev)  # regular entry point (library-owned scratch)
            gpu.sync()
            uold = C.c_void_p()
            assert L.rh_state_ptrs(C.byref(uold), None, None, None) == 0
            out.fill_(-1.0)
            torch.cuda.synchronize()
            rc = f(uold, int(m.noct[lev]), None, dx, P.gamma, P.smallr, P.smallc, P.courant_factor,
                   grav.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(out.data_ptr()), None)
            assert rc == 0, L.rh_last_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            np.testing.assert_allclose(got[[0, 1, 2, 4]], expected[[0, 1, 2, 4]], rtol=1e-12)
            assert got[3] == 0.0
            gpu.step_uniform()  # new state for the second call
            gpu.sync()
    finally:
        gpu.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = lib()
    f = _bind(L)
    grav = np.zeros(3)
    dummy = C.c_void_p(16)  # never dereferenced: the size check fails first
    rc = f(dummy, 2097152 + 1, None, 0.1, 1.4, 1e-10, 1e-10, 0.8, grav.ctypes.data_as(C.POINTER(C.c_double)),
           C.c_void_p(16), None)
    assert rc != 0
    assert "num_octs" in L.rh_last_error().decode()
