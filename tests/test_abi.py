"""The C-ABI library builds, loads and exports every symbol its headers declare
(no compute calls: these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

from ramses2_b200 import build as rb
from ramses2_b200._lib import LIB_PATH, RHError, check, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in ("ramses_hydro.h", "ramses_hydro_ext.h", "ramses_hydro_batch.h", "ramses_hydro_io.h"):
        p = os.path.join(ROOT, "include", h)
        if not os.path.exists(p):
            continue
        src = open(p).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char\*|double|long long|void)\s+\**\s*(rh_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_builds_and_loads():
    rb.build()
    assert os.path.exists(LIB_PATH)
    L = lib()
    assert L is not None


def test_every_declared_symbol_is_exported():
    L = lib()
    names = declared_symbols()
    assert len(names) >= 32, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_calls_before_init_report_state_errors():
    L = lib()
    # no device work: these fail fast on the host
    rc = L.rh_set_unew(1, 8)
    assert rc != 0
    assert "rh_init" in L.rh_last_error().decode()
    with pytest.raises(RHError):
        check(rc, "rh_set_unew")


def test_ext_tile_registry_lists_compiled_shapes():
    L = lib()
    tx = (C.c_int * 16)()
    ty = (C.c_int * 16)()
    mb = (C.c_int * 16)()
    n = L.rh_list_tiles(0, tx, ty, mb, 16)
    shapes = {(tx[i], ty[i]) for i in range(min(n, 16))}
    assert (7, 7) in shapes and (8, 8) in shapes
    n32 = L.rh_list_tiles(1, tx, ty, mb, 16)
    assert n32 >= 3
    assert {mb[i] for i in range(min(n32, 16))} >= {1, 2}


def test_batch_calls_before_init_report_state_errors():
    from ramses2_b200._abi import BatchIC, BatchProblem

    L = lib()
    assert L.rh_batch_init(0, 2, 3, 1024) == 4  # RH_ESTATE: rh_init not called
    pid = C.c_int()
    p, ic = BatchProblem(), BatchIC()
    assert L.rh_batch_add(C.byref(p), C.byref(ic), C.byref(pid)) == 4
    assert L.rh_batch_step(1) == 4
    assert L.rh_batch_free() == 0
