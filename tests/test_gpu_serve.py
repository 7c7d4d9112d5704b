"""Serving loop (ramses2_b200/serve.py): requests admitted by HBM footprint
into one device-resident batch, continuous batching, and every result the
same as the request solved alone (bitwise: a problem's step never depends on
what else shares the launch)."""
import copy

import numpy as np
import pytest

from ramses2_b200.batch import Batch
from ramses2_b200.serve import BYTES_PER_OCT, HydroServer, make_requests

pytestmark = pytest.mark.gpu


def _solve_alone(precision, req):
    b = Batch(precision, pool_octs=(req.cells // 8) + 8)
    try:
        pid = b.add(req.prob, req.ic)
        for _ in range(1000):
            b.step(4)
            if b.status(pid)["done"]:
                break
        st = b.status(pid)
        return b.fetch(pid), st
    finally:
        b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_served_results_equal_alone(precision):
    reqs = make_requests(10, rate_hz=1e6, seed=7, steps=(6, 24), sides_2d=(32, 64), sides_3d=(16, 32))
    pool = 3 * 32 ** 3 // 8 * BYTES_PER_OCT[precision]  # room for a few problems at a time: forces queueing
    srv = HydroServer(precision, pool_bytes=pool, chunk=2)
    try:
        mine = [copy.copy(r) for r in reqs]
        stats = srv.run(mine, realtime=False)
        served = {r.rid: r for r in mine}
    finally:
        srv.close()
    assert stats["served"] == len(reqs) and stats["rejected"] == 0
    for r in reqs:
        got = served[r.rid]
        ref, st = _solve_alone(precision, r)
        assert got.nsteps == st["nstep"]
        assert got.t == st["t"]
        assert got.t == pytest.approx(r.prob.t_end, rel=1e-12) or got.nsteps == r.prob.max_steps
        assert np.array_equal(got.result, ref), r


def test_server_rejects_requests_larger_than_the_pool():
    reqs = make_requests(3, rate_hz=1e6, seed=3, frac_2d=0.0, steps=(4, 6), sides_3d=(32, 32))
    srv = HydroServer("fp32_bulk", pool_bytes=(32 ** 3 // 8) * BYTES_PER_OCT["fp32_bulk"] - 1, chunk=2)
    try:
        stats = srv.run(reqs, realtime=False)
    finally:
        srv.close()
    assert stats["rejected"] == 3 and stats["served"] == 0


def test_served_requests_leave_reference_layout_snapshots(tmp_path):
    """With snapshot_dir, each finished request leaves an output directory whose
    hydro file holds the request's final density (float32) and whose amr file
    lists its octs; info.txt carries its step count."""
    from ramses2_b200 import files

    reqs = make_requests(4, rate_hz=1e6, seed=3, steps=(4, 8), sides_2d=(32, 32), sides_3d=(16, 16))
    srv = HydroServer("fp64", pool_bytes=64 << 20, chunk=2, snapshot_dir=str(tmp_path))
    try:
        srv.run(reqs, realtime=False)
    finally:
        srv.close()
    for r in reqs:
        assert r.snapshot and sorted(__import__("os").listdir(r.snapshot)) == [
            "amr.00001", "hydro.00001", "hydro_header.txt", "info.txt"]
        hyd = files.parse_image(open(r.snapshot + "/hydro.00001", "rb").read(), "hydro_output")
        amr = files.parse_image(open(r.snapshot + "/amr.00001", "rb").read(), "amr")
        noct = r.cells // 8
        assert hyd["noct"] == {1: noct} and amr["noct"] == {1: noct}
        assert np.array_equal(hyd["levels"][1][:, 0, :], r.result[:, 0, :].astype(np.float32))
        assert "nstep_coarse=%11d" % r.nsteps in open(r.snapshot + "/info.txt").read()
