"""Build librh_b200.so (the sm_100a CUDA library) in-tree with nvcc.

Every ``csrc/*.cu`` is compiled to an object under ``_build/`` in parallel and
linked into ``ramses2_b200/librh_b200.so``; the library is rebuilt only when a
source or header is newer than it or the set of sources changed since the
last link (a deleted instantiation unit must not stay in the library).
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librh_b200.so")
STAMP = os.path.join(BUILD, "sources.txt")  # the sources of the last link, one name per line
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
         "-I", CSRC, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(CSRC, "*.inc")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    if not all(os.path.getmtime(d) <= t for d in _deps()):
        return False
    try:
        with open(STAMP) as f:
            linked = f.read().split()
    except OSError:
        return True  # a library shipped without its build folder
    return linked == [os.path.basename(s) for s in _sources()]


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(force=False, verbose=False, jobs=None, ptxas_info=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = jobs or min(16, os.cpu_count() or 4)
    objs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, log in ex.map(lambda s: _compile(s, extra), _sources()):
            objs.append(obj)
            if verbose and log:
                sys.stderr.write(log)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write("\n".join(os.path.basename(s) for s in _sources()) + "\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
