"""Small, fixed workloads for profiler captures (ncu) of the library's kernels.

Each case builds its input, runs the kernel a few times and exits 0; the
commands under ``profiles/`` name these cases, so every capture there can be
repeated from the repository alone:

    python -m ramses2_b200.profcase pencil <level> <fp64|fp32_bulk> <txo,tyo,minb,lz>
        uniform Sedov3D (outflow, gamma 1.4, moncen, HLLC) on a 2^level grid,
        tile set explicitly, three full steps (godunov_pencil*_kernel)
    python -m ramses2_b200.profcase batch <nproblems> <fp64|fp32_bulk>
        the first n problems of the seeded Riemann/blast ensemble in one
        persistent launch per step, four timed steps (batch_step_kernel)
    python -m ramses2_b200.profcase plane2d
        16 2D blasts of sides 1024..256 on the plane tile body, FP32-bulk
    python -m ramses2_b200.profcase amr <fp64|fp32_bulk>
        Sedov on levels 7-10 (hydro_refine gradient criteria), four coarse steps
"""
import sys


def pencil(level, prec, tile):
    from ramses2_b200._abi import HydroParams
    from ramses2_b200.hydro import GodunovGPU
    from ramses2_b200.mesh import sedov3d, uniform_mesh

    tx, ty, mb, lz = (int(x) for x in tile.split(","))
    m = uniform_mesh(int(level), nsubgrid=1, bc="outflow")
    sedov3d(m)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    g = GodunovGPU(m, P, precision=prec)
    g.set_tile(tx, ty, lz, mb)
    for _ in range(3):
        g.step_uniform()
    g.sync()
    g.close()
    print("ok")


def batch(n, prec):
    from ramses2_b200.batch import Batch, ensemble_octs, riemann_blast_ensemble

    ens = riemann_blast_ensemble(int(n))
    b = Batch(prec, slope_type=2, riemann="hllc", pool_octs=ensemble_octs(ens) + 64)
    for p, ic in ens:
        p.max_steps = 1 << 30
        b.add(p, ic)
    b.set_tile(*((7, 7, 2, 32) if prec == "fp32_bulk" else (8, 4, 2, 32)))
    ms = b.bench(4)
    print("ms/step %.3f  G cell-updates/s %.2f" % (ms, ensemble_octs(ens) * 8 / ms / 1e6))
    b.close()


def plane2d():
    from ramses2_b200.batch import Batch, ic_blast, problem

    b = Batch("fp32_bulk", pool_octs=1 << 22)
    for s in (1024, 768, 512, 256) * 4:
        b.add(problem((s, s, 2), dx=1.0 / s, ndim=2, bc=["outflow"] * 4 + ["periodic"] * 2, t_end=1e9),
              ic_blast([1.0, 0, 0, 0, 1e-3], 10.0, 0.05, [0.5, 0.5, 0.0]))
    b.step(2)
    print("ms", b.bench(3))
    b.close()


def amr(prec):
    from ramses2_b200._abi import HydroParams
    from ramses2_b200.hydro import GodunovGPU
    from ramses2_b200.mesh import sedov_amr_mesh

    m, g = sedov_amr_mesh(7, 10, radius=0.08)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                         interpol_type=1)
    gpu = GodunovGPU(m, P, precision=prec)
    for _ in range(4):
        gpu.coarse_step()
    gpu.sync()
    gpu.close()
    print("ok")


CASES = {"pencil": pencil, "batch": batch, "plane2d": plane2d, "amr": amr}

if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1] not in CASES:
        sys.exit(__doc__)
    CASES[sys.argv[1]](*sys.argv[2:])
