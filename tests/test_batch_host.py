"""Host-side pieces of the batch runtime (no GPU): the reference-layout oct
packing of dense boxes and the problem footprint the admission uses."""
import ctypes as C

import numpy as np

from ramses2_b200.batch import dense_to_octs, octs_to_dense, problem
from ramses2_b200._lib import lib


def test_octs_layout_round_trip():
    a = np.random.default_rng(0).standard_normal((5, 6, 4, 8))
    assert np.array_equal(octs_to_dense(dense_to_octs(a), (8, 4, 6)), a)


def test_octs_layout_cell_order_is_the_reference_oct_order():
    # cell c of an oct sits at (c & 1, (c >> 1) & 1, c >> 2) (x fastest), octs row-major
    n = (4, 6, 2)
    z, y, x = np.indices((n[2], n[1], n[0]))
    a = np.stack([x, y, z, x + 10 * y + 100 * z, np.zeros_like(x)]).astype(np.float64)
    o = dense_to_octs(a)
    nxo, nyo = n[0] // 2, n[1] // 2
    for oct_ in range(o.shape[0]):
        ox, oy, oz = oct_ % nxo, (oct_ // nxo) % nyo, oct_ // (nxo * nyo)
        for c in range(8):
            assert o[oct_, 0, c] == 2 * ox + (c & 1)
            assert o[oct_, 1, c] == 2 * oy + ((c >> 1) & 1)
            assert o[oct_, 2, c] == 2 * oz + (c >> 2)


def test_footprint_counts_both_time_levels():
    L = lib()
    p = problem((32, 16, 8))
    # before rh_batch_init the footprint is that of the FP64 layout: 2 x 320 B per oct
    assert L.rh_batch_footprint(C.byref(p)) == (16 * 8 * 4) * 640


def test_request_stream_shapes_and_arrivals():
    from ramses2_b200.serve import make_requests

    reqs = make_requests(200, rate_hz=5.0, seed=1)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    # Poisson: mean gap 1/rate within sampling error
    assert abs(np.diff(arr).mean() - 0.2) < 0.05
    kinds = {r.kind for r in reqs}
    assert kinds == {"sedov2d", "interface2d", "sedov3d"}
    for r in reqs:
        n = list(r.prob.n)
        if r.prob.ndim == 2:
            assert n[2] == 2 and 64 <= n[0] == n[1] <= 1024
        else:
            assert 32 <= n[0] == n[1] == n[2] <= 192
        assert all(v % 2 == 0 for v in n)
        assert r.prob.t_end > 0 and 20 <= r.target_steps <= 400 and r.prob.max_steps == 400


def test_initial_dt_is_the_courant_formula():
    import math

    from ramses2_b200.serve import initial_dt

    q = [1.0, 0.5, 0.0, 0.0, 1.0]
    g, dx, C = 1.4, 0.01, 0.8
    c = math.sqrt(g)
    want = 2 * C * dx / ((0.5 + c + c + c) * (1 + math.sqrt(1 + 2 * C * 1e-4)))
    assert initial_dt([q], g, dx, 3, C) == want
