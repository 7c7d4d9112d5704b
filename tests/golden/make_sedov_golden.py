"""Generate tests/golden/sedov_analytic_3d.npz from the reference's own
analytic Sedov solver (utils/py/sedov.py:4 sedovana), imported from the
read-only reference checkout (argument, else REF_ROOT, else oracle/Makefile's
REF_ROOT).  Run where the checkout exists:

    python tests/golden/make_sedov_golden.py [reference-root]

The fixture holds the dimensionless self-similar profiles (r, d, u, p) for
gamma = 1.4 and 1.6667 in 3D; scale with (E/rho0)^(1/5) t^(2/5) etc. as the
sedovana docstring describes.
"""
import os
import sys

import numpy as np


def main(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "utils", "py"))
    from sedov import sedovana  # the reference's analytic solver

    out = {}
    for g in (1.4, 1.6667):
        r, d, u, p = sedovana(gamma=g, dim=3, n1=2000, n2=2000)
        key = str(g).replace(".", "p")
        out["r_" + key] = r
        out["d_" + key] = d
        out["u_" + key] = u
        out["p_" + key] = p
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "sedov_analytic_3d.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        root = sys.argv[1]
    else:
        here = os.path.dirname(os.path.abspath(__file__))
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(here)), "oracle"))
        import oracle

        root = oracle.reference_root()
    if root is None:
        sys.exit("reference checkout not found: set REF_ROOT or pass its path")
    main(root)
