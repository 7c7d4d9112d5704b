"""The ABI driven from plain C (the role the Fortran host plays): the example
host in tests/c_host compiles with gcc against include/ and links to
librh_b200.so; without a GPU it reports "no device", on a B200 it runs ten
Sedov steps and checks mass conservation."""
import os
import subprocess

import pytest

from ramses2_b200 import build as rb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    lib = rb.build()
    exe = str(tmp_path / "sedov_host")
    subprocess.run(["gcc", "-O2", "-std=c99", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_host", "sedov_host.c"), "-o", exe,
                    "-L", os.path.dirname(lib), "-lrh_b200", "-Wl,-rpath," + os.path.dirname(lib), "-lm"],
                   check=True)
    return exe


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="the GPU variant runs under -m gpu")
def test_c_host_builds_and_reports_no_device(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "no device" in r.stdout


@pytest.mark.gpu
def test_c_host_runs_sedov_and_conserves_mass(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "relative drift" in r.stdout
