"""Restart and snapshot files (include/ramses_hydro_io.h) on the CPU: the
oracle's restatement of the reference's writers against the golden images
that the reference's own Python reader decoded (tests/golden/make_io_golden.py),
the live reference reader where the checkout exists, the restart reader's
offset formulas, and the text files of an output directory."""
import importlib.util
import os

import numpy as np
import pytest

import oracle
from ramses2_b200 import files
from ramses2_b200._abi import OCT_DTYPE
from ramses2_b200.mesh import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "io_amr3to5.npz")
_REF = oracle.reference_root()
REF_IO = os.path.join(_REF, "utils", "py", "ramses_io.py") if _REF else ""


def fixture_mesh():
    """The golden mesh: oct records from the fixture, uold = the backup payload."""
    z = np.load(GOLD)
    grid = np.zeros(len(z["lev"]), OCT_DTYPE)
    grid["ckey"], grid["refined"], grid["lev"] = z["ckey"], z["refined"], z["lev"]
    m = Mesh(grid, int(z["levelmin"]), int(z["levelmax"]), bc="periodic")
    nlev = m.levelmax - m.levelmin + 1
    m.uold[:] = np.frombuffer(z["img_hydro_backup"].tobytes(), "<f8", offset=16 + 4 * nlev).reshape(-1, 5, 8)
    return m, z


def test_output_prims_restate_the_reference_expressions():
    # numpy evaluates each operation IEEE-rounded, in the order written in
    # hydro/output_hydro.f90:86-130, with no contraction
    m, z = fixture_mesh()
    u = m.uold
    d = u[:, 0]
    vx, vy, vz = u[:, 1] / d, u[:, 2] / d, u[:, 3] / d
    ekin = 0.5 * d * (vx * vx + vy * vy + vz * vz)
    p = (float(z["gamma"]) - 1) * (u[:, 4] - ekin - 0.0 - 0.0)
    ref = np.stack([d, vx, vy, vz, p], axis=1).astype(np.float32)
    q = oracle.output_prims(u, float(z["gamma"]))
    assert q.tobytes() == ref.tobytes()


@pytest.mark.parametrize("kind,key", [(1, "img_amr"), (2, "img_hydro_backup"), (3, "img_hydro_output")])
def test_oracle_images_match_golden(kind, key):
    m, z = fixture_mesh()
    img = oracle.file_image(kind, m.uold, m.grid, m.head, m.noct, m.levelmin, m.levelmax, float(z["gamma"]))
    assert img == z[key].tobytes()


def test_golden_images_decode_as_the_reference_reader_did():
    """What the reference's ramses_io returned for these bytes (stored in the
    fixture) equals the package's own decoding and the mesh."""
    m, z = fixture_mesh()
    amr = files.parse_image(z["img_amr"].tobytes(), "amr")
    out = files.parse_image(z["img_hydro_output"].tobytes(), "hydro_output")
    bak = files.parse_image(z["img_hydro_backup"].tobytes(), "hydro_backup")
    assert list(z["ref_levels"]) == list(range(m.levelmin, m.levelmax + 1))
    assert list(z["ref_noct"]) == [int(m.noct[l]) for l in z["ref_levels"]]
    assert list(z["ref_var_names"]) == ["density", "velocity_x", "velocity_y", "velocity_z", "thermal_pressure"]
    for l in z["ref_levels"]:
        sl = m.level_slice(l)
        ck, bits = amr["levels"][l]
        assert np.array_equal(z["ref_ckey_%d" % l], ck)
        assert np.array_equal(ck, m.grid["ckey"][sl])
        assert np.array_equal(z["ref_bits_%d" % l], bits)
        refined = ((bits[:, None] >> np.arange(8)) & 1).astype(bool)
        assert np.array_equal(refined, m.grid["refined"][sl] != 0)
        assert z["ref_prim_%d" % l].tobytes() == out["levels"][l].tobytes()
        assert bak["levels"][l].tobytes() == m.uold[sl].tobytes()
    # leaf cells: every unrefined cell once, with its density
    nleaf = sum(int((m.grid["refined"][m.level_slice(l)] == 0).sum()) for l in z["ref_levels"])
    assert len(z["ref_leaf_density"]) == nleaf
    rho = np.concatenate([out["levels"][l][:, 0][m.grid["refined"][m.level_slice(l)] == 0]
                          for l in z["ref_levels"]])
    assert np.array_equal(np.sort(z["ref_leaf_density"]), np.sort(rho))
    assert np.allclose(z["ref_info"], [1.0, 0.125, 1.4, 7])


@pytest.mark.skipif(not os.path.exists(REF_IO), reason="reference checkout absent")
def test_live_reference_reader(tmp_path):
    """The reference's reader reads an output directory written by the package
    (text files) from oracle images; info.txt values round-trip."""
    spec = importlib.util.spec_from_file_location("ref_ramses_io", REF_IO)
    rio = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rio)
    m, z = fixture_mesh()
    g = float(z["gamma"])
    img = {k: oracle.file_image(k, m.uold, m.grid, m.head, m.noct, m.levelmin, m.levelmax, g) for k in (1, 3)}
    path = files.dir_name(str(tmp_path), 42)
    info = files.info_txt(m.levelmin, m.levelmax, m.ngridmax, 11, m.boxlen, 0.3125, g)
    files.write_dir(path, img[1], img[3], info, backup=False)
    o = rio.Output(path)
    assert o.info["time"] == 0.3125 and o.info["nstep_coarse"] == 11 and o.info["gamma"] == g
    for l in o.levels():
        assert o.grid["hydro"][0].read_level(l).tobytes() == oracle.output_prims(m.uold[m.level_slice(l)],
                                                                                  g).tobytes()
    c = rio.leaf_cells(path)
    assert c.ncell == len(z["ref_leaf_density"])


def test_restart_offsets_match_the_images():
    """Level offsets the restart reader computes (init_refine_restart.f90:387,396)
    point at each level's first record in the images."""
    m, z = fixture_mesh()
    nlev = m.levelmax - m.levelmin + 1
    for kind, key, rec in ((1, "img_amr", 16), (2, "img_hydro_backup", 320)):
        off = oracle.restart_offsets(kind, m.levelmin, m.levelmax, m.noct)
        b = z[key].tobytes()
        hs = (12 if kind == 1 else 16) + 4 * nlev
        assert off[m.levelmin] == hs
        for l in range(m.levelmin, m.levelmax + 1):
            a = int(m.head[l]) - 1
            first = b[off[l]:off[l] + rec]
            if kind == 1:
                r = np.frombuffer(first, "<i4")
                assert list(r[:3]) == list(m.grid["ckey"][a])
            else:
                assert first == m.uold[a].tobytes()


def test_text_files():
    assert files.fortran_e(1.0) == "  0.100000000000000E+01"
    assert files.fortran_e(0.0) == "  0.000000000000000E+00"
    assert files.fortran_e(-1.5e-7) == " -0.150000000000000E-06"
    assert files.fortran_e(1.4) == "  0.140000000000000E+01"
    info = files.info_txt(7, 10, 1000, 3, 1.0, 0.25, 1.4)
    lines = info.splitlines()
    assert lines[0] == "nfile       =          1"
    assert lines[4] == "levelmax    =         10"
    assert lines[6] == "nstep_coarse=          3"
    assert lines[7] == ""
    assert lines[9] == "time        =  0.250000000000000E+00"
    h = files.hydro_header_txt(backup=False).splitlines()
    assert h == ["nvar        =          5", "variable # 1: density", "variable # 2: velocity_x",
                 "variable # 3: velocity_y", "variable # 4: velocity_z", "variable # 5: thermal_pressure"]
    assert files.hydro_header_txt(backup=True).splitlines()[5] == "variable # 5: total_energy"


def test_parse_rejects_inconsistent_images():
    m, z = fixture_mesh()
    b = z["img_hydro_backup"].tobytes()
    with pytest.raises(ValueError):
        files.parse_image(b[:-8], "hydro_backup")
    with pytest.raises(ValueError):
        files.parse_image(b, "hydro_output")
