"""Restart and snapshot file images made by the CUDA library
(include/ramses_hydro_io.h) against the oracle's restatement of the
reference's writers: byte-identical images of the golden mesh, of stepped AMR
and uniform states in FP64 and FP32-bulk, of batch problems; restart
(rh_restore_hydro) brings back the backed-up state bit for bit."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from ramses2_b200 import files
from ramses2_b200._abi import OCT_DTYPE, HydroParams
from ramses2_b200.batch import Batch, ic_split, problem
from ramses2_b200.hydro import GodunovGPU, amr_coarse_step
from ramses2_b200.mesh import Mesh, sedov3d, uniform_mesh

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "io_amr3to5.npz")
KINDS = (files.FILE_AMR, files.FILE_HYDRO_BACKUP, files.FILE_HYDRO_OUTPUT)


def fixture_mesh():
    z = np.load(GOLD)
    grid = np.zeros(len(z["lev"]), OCT_DTYPE)
    grid["ckey"], grid["refined"], grid["lev"] = z["ckey"], z["refined"], z["lev"]
    m = Mesh(grid, int(z["levelmin"]), int(z["levelmax"]), bc="periodic")
    nlev = m.levelmax - m.levelmin + 1
    m.uold[:] = np.frombuffer(z["img_hydro_backup"].tobytes(), "<f8", offset=16 + 4 * nlev).reshape(-1, 5, 8)
    return m, z


def params(gamma=1.4):
    P = HydroParams()
    P.gamma, P.smallr, P.smallc, P.courant_factor = gamma, 1e-10, 1e-10, 0.8
    P.slope_type, P.riemann = 2, 3
    return P


def oracle_image(kind, m, uold, gamma):
    return oracle.file_image(kind, uold, m.grid, m.head, m.noct, m.levelmin, m.levelmax, gamma)


def test_golden_images_fp64():
    m, z = fixture_mesh()
    g = GodunovGPU(m, params(float(z["gamma"])), "fp64")
    try:
        assert g.file_image("amr") == z["img_amr"].tobytes()
        assert g.file_image("hydro_backup") == z["img_hydro_backup"].tobytes()
        assert g.file_image("hydro_output") == z["img_hydro_output"].tobytes()
    finally:
        g.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_stepped_amr_images_match_oracle(precision):
    m, z = fixture_mesh()
    gamma = float(z["gamma"])
    g = GodunovGPU(m, params(gamma), precision)
    try:
        for _ in range(2):
            amr_coarse_step(g, m)
        u = g.fetch_uold()  # FP32-bulk: float32 values widened exactly
        for kind in KINDS:
            assert g.file_image(kind) == oracle_image(kind, m, u, gamma), kind
    finally:
        g.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_restart_restores_state_bitwise(precision, tmp_path):
    m = uniform_mesh(5, bc="outflow")
    sedov3d(m, gamma=1.4)
    g = GodunovGPU(m, params(), precision)
    try:
        g.step_uniform()
        path = g.write_output(str(tmp_path), 3, time=0.5, nstep_coarse=1, backup=True)
        u0 = g.fetch_uold()
        g.restore(path)  # a restart point: the CFL caches start empty
        assert np.array_equal(g.fetch_uold(), u0)
        g.step_uniform()
        dt_ref, _ = g.step_uniform()
        u_ref = g.fetch_uold()
        assert not np.array_equal(u_ref, u0)
        g.restore(path)
        assert np.array_equal(g.fetch_uold(), u0)
        g.step_uniform()
        dt2, _ = g.step_uniform()
        assert dt2 == dt_ref
        assert np.array_equal(g.fetch_uold(), u_ref)
        # the directory holds the reference's four files
        assert sorted(os.listdir(path)) == ["amr.00001", "hydro.00001", "hydro_header.txt", "info.txt"]
        with open(os.path.join(path, "hydro.00001"), "rb") as f:
            assert f.read() == oracle_image(files.FILE_HYDRO_BACKUP, m, u0, 1.4)
    finally:
        g.close()


def test_restore_rejects_a_foreign_image():
    m = uniform_mesh(4)
    sedov3d(m, gamma=1.4)
    g = GodunovGPU(m, params(), "fp64")
    try:
        other = uniform_mesh(3)
        img = oracle_image(files.FILE_HYDRO_BACKUP, other, other.uold, 1.4)
        with pytest.raises(RuntimeError):
            g.restore(img)
        good = g.file_image("hydro_backup")
        with pytest.raises(RuntimeError):
            g.restore(good[:-8])
        g.restore(good)
    finally:
        g.close()


def test_device_image_equals_host_image():
    from cuda.bindings import runtime as rt
    m = uniform_mesh(4)
    sedov3d(m, gamma=1.4)
    g = GodunovGPU(m, params(), "fp32_bulk")
    try:
        g.step_uniform()
        host = g.file_image("hydro_output")
        ptr, n = C.c_void_p(), C.c_longlong()
        assert g.L.rh_file_image_device(files.FILE_HYDRO_OUTPUT, 1.4, C.byref(ptr), C.byref(n)) == 0
        assert n.value == len(host)
        out = np.empty(n.value, np.uint8)
        err, = rt.cudaMemcpy(out.ctypes.data, ptr.value, n.value, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert int(err) == 0
        assert out.tobytes() == host
    finally:
        g.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
def test_batch_problem_images(precision, tmp_path):
    b = Batch(precision, pool_octs=1 << 16)
    try:
        n = (16, 12, 8)
        p = problem(n, gamma=1.6, t_end=10.0, max_steps=3)
        pid = b.add(p, ic_split(0, [1.0, 0.5, 0.0, 0.0, 1.0], [0.125, 0.0, 0.1, 0.0, 0.1]))
        b.step(3)
        u = b.fetch(pid)
        nxo, nyo, nzo = n[0] // 2, n[1] // 2, n[2] // 2
        grid = np.zeros(nxo * nyo * nzo, OCT_DTYPE)
        o = np.arange(len(grid))
        grid["ckey"][:, 0], grid["ckey"][:, 1], grid["ckey"][:, 2] = o % nxo, (o // nxo) % nyo, o // (nxo * nyo)
        grid["lev"] = 1
        head, noct = np.array([0, 1]), np.array([0, len(grid)])
        for kind in KINDS:
            assert b.file_image(pid, kind) == oracle.file_image(kind, u, grid, head, noct, 1, 1, 1.6), kind
        path = b.write_output(pid, str(tmp_path), 1)
        info = open(os.path.join(path, "info.txt")).read()
        assert "nstep_coarse=          3" in info
    finally:
        b.close()
