"""Generates tests/golden/io_amr3to5.npz: restart and snapshot file images of a
small three-level mesh, made by the oracle's restatement of the reference's
writers and decoded by the reference's own Python reader
(utils/py/ramses_io.py of the reference checkout: Output, GridFile.read_amr,
GridFile.read_level, leaf_cells).

Run from the repository root with the reference checkout at REF_ROOT
(default: oracle/Makefile's REF_ROOT):

    python tests/golden/make_io_golden.py

The fixture holds the inputs (oct records; uold is the backup image's
payload), the three images and what
the reference's reader returned for the output directory; tests compare the
oracle and the CUDA library against it without the reference present.
"""
import importlib.util
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from ramses2_b200 import files  # noqa: E402
from ramses2_b200.mesh import amr_mesh, fill_amr_prim  # noqa: E402

GAMMA = 1.4
OUT = os.path.join(ROOT, "tests", "golden", "io_amr3to5.npz")


def golden_mesh():
    """Levels 3..5 around a sphere, seeded smooth primitive fields."""
    m = amr_mesh(3, 5, lambda x, l: np.sqrt(((x - 0.52) ** 2).sum(-1)) < 0.2, bc="periodic")
    rng = np.random.default_rng(20261203)
    k = rng.uniform(1.0, 3.0, size=(5, 3))
    ph = rng.uniform(0.0, 2 * np.pi, size=5)

    def prim(x, lev):
        w = [np.sin(2 * np.pi * (x @ k[i]) + ph[i]) for i in range(5)]
        return 1.0 + 0.5 * w[0], 0.7 * w[1], -0.4 * w[2], 0.3 * w[3], 0.5 + 0.25 * w[4]

    fill_amr_prim(m, prim, GAMMA)
    return m


def ramses_io(ref_root):
    path = os.path.join(ref_root, "utils", "py", "ramses_io.py")
    spec = importlib.util.spec_from_file_location("ref_ramses_io", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def images(m):
    return {k: oracle.file_image(v, m.uold, m.grid, m.head, m.noct, m.levelmin, m.levelmax, GAMMA)
            for k, v in (("amr", 1), ("hydro_backup", 2), ("hydro_output", 3))}


def read_with_reference(rio, m, img, time=0.125, nstep=7):
    """Write an output directory from the images and read it back with the
    reference's reader."""
    with tempfile.TemporaryDirectory() as tmp:
        path = files.dir_name(tmp, 1)
        info = files.info_txt(m.levelmin, m.levelmax, m.ngridmax, nstep, m.boxlen, time, GAMMA)
        files.write_dir(path, img["amr"], img["hydro_output"], info, backup=False)
        o = rio.Output(path)
        out = {"ref_levels": np.array(o.levels()),
               "ref_noct": np.array([o.noct_per_level()[l] for l in o.levels()]),
               "ref_var_names": np.array(o.var_names["hydro"]),
               "ref_info": np.array([o.info["boxlen"], o.info["time"], o.info["gamma"], o.info["nstep_coarse"]])}
        for l in o.levels():
            ck, bits = o.grid["amr"][0].read_amr(l)
            out["ref_ckey_%d" % l] = np.asarray(ck)
            out["ref_bits_%d" % l] = np.asarray(bits)
            out["ref_prim_%d" % l] = np.asarray(o.grid["hydro"][0].read_level(l))
        c = rio.leaf_cells(path)
        out["ref_leaf_level"] = np.asarray(c.level)
        out["ref_leaf_icell"] = np.asarray(c.icell)
        out["ref_leaf_density"] = np.asarray(c["density"])
        out["ref_leaf_pressure"] = np.asarray(c["thermal_pressure"])
    return out


def main():
    ref_root = oracle.reference_root()
    if ref_root is None:
        sys.exit("reference checkout not found: set REF_ROOT")
    rio = ramses_io(ref_root)
    m = golden_mesh()
    img = images(m)
    dec = read_with_reference(rio, m, img)
    np.savez_compressed(
        OUT, ckey=m.grid["ckey"], refined=m.grid["refined"], lev=m.grid["lev"], head=m.head,
        noct=m.noct, levelmin=m.levelmin, levelmax=m.levelmax, gamma=GAMMA,
        img_amr=np.frombuffer(img["amr"], np.uint8), img_hydro_backup=np.frombuffer(img["hydro_backup"], np.uint8),
        img_hydro_output=np.frombuffer(img["hydro_output"], np.uint8), **dec)
    print(OUT, {k: len(v) for k, v in img.items()})


if __name__ == "__main__":
    main()
