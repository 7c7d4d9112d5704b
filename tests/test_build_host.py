"""The in-tree build's staleness rule (ramses2_b200/build.py), on a scratch
tree: the library is relinked when a source or header is newer than it, or
when the set of CUDA sources differs from the one of its last link (a
deleted instantiation unit must not stay in the library)."""
import os
import time

import ramses2_b200.build as B


def _tree(tmp_path, monkeypatch, names):
    csrc = tmp_path / "pkg" / "csrc"
    inc = tmp_path / "include"
    csrc.mkdir(parents=True)
    inc.mkdir()
    for n in names:
        (csrc / n).write_text("// %s\n" % n)
    (csrc / "k.cuh").write_text("// header\n")
    (inc / "api.h").write_text("/* api */\n")
    lib = tmp_path / "pkg" / "lib.so"
    build = tmp_path / "pkg" / "_build"
    build.mkdir()
    monkeypatch.setattr(B, "ROOT", str(tmp_path))
    monkeypatch.setattr(B, "CSRC", str(csrc))
    monkeypatch.setattr(B, "LIB", str(lib))
    monkeypatch.setattr(B, "BUILD", str(build))
    monkeypatch.setattr(B, "STAMP", str(build / "sources.txt"))
    return csrc, lib, build


def _link(lib, build, names):
    """What build() leaves behind: the library, newer than every source, and
    the stamp of the sources it linked."""
    later = time.time() + 10
    lib.write_bytes(b"\x7fELF")
    os.utime(lib, (later, later))
    (build / "sources.txt").write_text("\n".join(sorted(names)) + "\n")


def test_fresh_library_is_up_to_date(tmp_path, monkeypatch):
    names = ["a.cu", "b.cu"]
    _, lib, build = _tree(tmp_path, monkeypatch, names)
    assert not B.up_to_date()  # no library yet
    _link(lib, build, names)
    assert B.up_to_date()


def test_newer_header_makes_it_stale(tmp_path, monkeypatch):
    names = ["a.cu", "b.cu"]
    csrc, lib, build = _tree(tmp_path, monkeypatch, names)
    _link(lib, build, names)
    later = os.path.getmtime(lib) + 5
    os.utime(csrc / "k.cuh", (later, later))
    assert not B.up_to_date()


def test_deleted_source_makes_it_stale(tmp_path, monkeypatch):
    names = ["a.cu", "b.cu", "c.cu"]
    csrc, lib, build = _tree(tmp_path, monkeypatch, names)
    _link(lib, build, names)
    assert B.up_to_date()
    os.remove(csrc / "c.cu")  # nothing is newer than the library now
    assert not B.up_to_date()


def test_added_source_makes_it_stale(tmp_path, monkeypatch):
    names = ["a.cu"]
    csrc, lib, build = _tree(tmp_path, monkeypatch, names)
    _link(lib, build, names)
    (csrc / "z.cu").write_text("// new\n")
    os.utime(csrc / "z.cu", (0, 0))  # older than the library
    assert not B.up_to_date()


def test_shipped_library_without_build_folder_is_kept(tmp_path, monkeypatch):
    names = ["a.cu"]
    _, lib, build = _tree(tmp_path, monkeypatch, names)
    _link(lib, build, names)
    os.remove(build / "sources.txt")
    assert B.up_to_date()
