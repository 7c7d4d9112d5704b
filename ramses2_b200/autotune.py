"""Autotuner of the Godunov pencil kernel.

Chooses, for one resident mesh and precision, the compiled tile shape
(txo x tyo octs), the register budget (1 or 2 CTAs per SM) and the pencil depth
(oct layers per CTA) by timing each candidate on the device with CUDA events
(rh_bench_godunov: back-to-back launches on the library stream, state larger
than L2).  The time of one candidate is the median of ``reps`` measurements.
"""
import itertools
import json
import os

import numpy as np

DEFAULT_LZ = (16, 24, 32, 40)


def tune(gpu, level, dt, lz_choices=DEFAULT_LZ, nrep=6, reps=3, log=None):
    """Pick the fastest (txo, tyo, minb, lz) for ``gpu`` (a GodunovGPU or a
    batch solver exposing tiles()/set_tile()/bench_godunov()).  Leaves the
    winner selected and returns (best, table)."""
    table = []
    for (tx, ty, mb), lz in itertools.product(gpu.tiles(), lz_choices):
        gpu.set_tile(tx, ty, lz, mb)
        gpu.bench_godunov(level, 2, dt)  # warm-up (tables, caches, clocks)
        ms = float(np.median([gpu.bench_godunov(level, nrep, dt) for _ in range(reps)]))
        table.append({"txo": tx, "tyo": ty, "minb": mb, "lz": lz, "ms": ms})
        if log:
            log("autotune %dx%d minb=%d lz=%d: %.3f ms" % (tx, ty, mb, lz, ms))
    best = min(table, key=lambda r: r["ms"])
    gpu.set_tile(best["txo"], best["tyo"], best["lz"], best["minb"])
    return best, table


def save(path, key, best, table):
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = {"best": best, "table": table}
    with open(path, "w") as f:
        json.dump(data, f, indent=1)
