"""The pencil kernels' FP64 reciprocal and square root (vrcp, vsqrt in
ramses2_b200/csrc/rh_vec.cuh: hardware estimates refined by Newton-Raphson
steps) against correctly rounded results, on the device: within 2 ulp of
CUDA's 1.0/x and sqrt(x) (which equal IEEE's, checked against numpy) over a
million positive normal doubles spanning 2^-1000 .. 2^1000, the range of every
density, pressure and sound-speed argument of the hydro step."""
import ctypes as C

import numpy as np
import pytest

from ramses2_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def ulps(a, b):
    """Distance in units in the last place between positive doubles."""
    return np.abs(a.view(np.int64) - b.view(np.int64))


def test_vrcp_vsqrt_within_two_ulp_of_correct_rounding():
    import torch

    L = lib()
    check(L.rh_init(0), "rh_init")
    rng = np.random.default_rng(2026)
    n = 1 << 20
    x = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-1000, 1000, n))
    x[:64] = np.ldexp(1.0, np.arange(-32, 32))              # exact powers of two
    x[64:128] = 1.0 + np.arange(64) * np.finfo(np.float64).eps  # just above 1
    x[128:192] = np.nextafter(np.ldexp(1.0, np.arange(-32, 32)), 0)  # just below powers of two
    dx = torch.from_numpy(x).to("cuda")
    out = torch.empty(4 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    check(L.rh_selftest_vmath(C.c_void_p(dx.data_ptr()), n, C.c_void_p(out.data_ptr())), "rh_selftest_vmath")
    o = out.cpu().numpy().reshape(4, n)
    rcp_ieee, sqrt_ieee = 1.0 / x, np.sqrt(x)
    assert np.array_equal(o[2], rcp_ieee) and np.array_equal(o[3], sqrt_ieee)  # CUDA's are correctly rounded
    ur, us = ulps(o[0], o[2]), ulps(o[1], o[3])
    assert ur.max() <= 2, (ur.max(), x[ur.argmax()])
    assert us.max() <= 2, (us.max(), x[us.argmax()])
