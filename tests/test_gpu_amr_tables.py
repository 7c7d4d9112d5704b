"""The device-side coarse-fine table builder (rh_amr_tables.cu) against the
host builder (build_amr_tables, rh_amr.cu): identical pencil headers, table
offsets, oct tables and interpolated ghost octs (sources, flip bits, fathers)
for every boundary type and two tiles; a mesh that is not properly nested is
rejected by both with the same message."""
import ctypes as C

import numpy as np
import pytest

from ramses2_b200._abi import HydroParams
from ramses2_b200._lib import lib
from ramses2_b200.hydro import GodunovGPU
from ramses2_b200.mesh import amr_mesh, sedov_amr_mesh

pytestmark = pytest.mark.gpu


def params():
    return HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                            interpol_type=1)


def tables(m, builder, amr_tile):
    g = GodunovGPU(m, params(), "fp64", amr_tile=amr_tile, table_builder=builder)
    L = lib()
    out = {}
    try:
        for l in range(m.levelmin, m.levelmax + 1):
            npen, ntab = C.c_int(), C.c_longlong()
            assert L.rh_level_info(l, C.byref(npen), C.byref(ntab)) == 0
            if npen.value == 0:
                continue
            phdr = np.zeros((npen.value, 4), np.int32)
            poff = np.zeros(npen.value, np.int64)
            tab = np.zeros(ntab.value, np.int32)
            assert L.rh_level_table(l, phdr.ctypes.data_as(C.POINTER(C.c_int)),
                                    poff.ctypes.data_as(C.POINTER(C.c_longlong)),
                                    tab.ctypes.data_as(C.POINTER(C.c_int)), ntab.value) == 0
            ng = L.rh_level_ghosts(l, None, None, None, 0)
            assert ng >= 0
            src = np.zeros((max(ng, 1), 7), np.int32)
            cf = np.zeros((max(ng, 1), 7), np.uint8)
            fa = np.zeros((max(ng, 1), 2), np.int32)
            assert L.rh_level_ghosts(l, src.ctypes.data_as(C.POINTER(C.c_int)),
                                     cf.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                     fa.ctypes.data_as(C.POINTER(C.c_int)), max(ng, 1)) == ng
            out[l] = (phdr, poff, tab, src[:ng], cf[:ng], fa[:ng])
    finally:
        g.close()
    return out


MESHES = {
    "sphere_outflow": lambda: amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.52) ** 2).sum(-1)) < 0.16, bc="outflow"),
    "sphere_periodic": lambda: amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.5) ** 2).sum(-1)) < 0.2, bc="periodic"),
    "slab_reflexive": lambda: amr_mesh(4, 6, lambda x, l: np.abs(x[:, 0] - 0.1) < 0.12, bc="reflexive"),
    "corner_outflow": lambda: amr_mesh(3, 6, lambda x, l: (x < 0.3).all(-1), bc="outflow"),
}


@pytest.mark.parametrize("amr_tile", [(8, 4, 2, 8), (4, 4, 2, 3)])
@pytest.mark.parametrize("name", sorted(MESHES))
def test_device_tables_equal_host_tables(name, amr_tile):
    m = MESHES[name]()
    host = tables(m, "host", amr_tile)
    dev = tables(m, "device", amr_tile)
    assert sorted(host) == sorted(dev) and host
    nghost = 0
    for l in host:
        for a, b, what in zip(host[l], dev[l], ("phdr", "poff", "tab", "gsrc_oct", "gsrc_cf", "gfather")):
            assert a.shape == b.shape and np.array_equal(a, b), (name, l, what)
        nghost += len(host[l][3])
    assert nghost > 0


def test_device_tables_on_amr_sedov_mesh():
    m, _ = sedov_amr_mesh(6, 8, radius=0.15)
    host = tables(m, "host", (8, 4, 2, 8))
    dev = tables(m, "device", (8, 4, 2, 8))
    for l in host:
        for a, b in zip(host[l], dev[l]):
            assert np.array_equal(a, b)


def test_unnested_mesh_rejected_by_both_builders():
    """A level-6 oct moved where level 5 has no octs: its neighbourhood cannot
    be interpolated, and both builders refuse the mesh."""
    from ramses2_b200.mesh import Mesh
    m = amr_mesh(4, 6, lambda x, l: np.sqrt(((x - 0.5) ** 2).sum(-1)) < 0.15, bc="outflow")
    bad = m.grid.copy()
    lev6 = np.nonzero(bad["lev"] == 6)[0]
    assert len(lev6) and not ((bad["lev"] == 5) & (bad["ckey"] < 3).all(axis=1)).any()
    bad["ckey"][lev6[0]] = (0, 0, 0)
    mb = Mesh(bad, m.levelmin, m.levelmax, bc="outflow")
    mb.uold[:] = 1.0
    L = lib()
    errs = []
    for builder in ("host", "device"):
        assert L.rh_init(0) == 0
        try:
            with pytest.raises(RuntimeError) as ei:
                GodunovGPU(mb, params(), "fp64", table_builder=builder)
            errs.append(str(ei.value))
        finally:
            L.rh_finalize()
    for e in errs:
        assert "level 6" in e and "not properly nested" in e, errs
