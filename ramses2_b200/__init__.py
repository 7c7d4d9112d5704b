"""B200-native RAMSES II Godunov hydro step.

The product is ``librh_b200.so`` (sm_100a CUDA, C ABI in ``include/``); this
package holds its Python host layer: mesh construction in the reference's
flat-oct layout (:mod:`.mesh`), the reference-shaped leaf calls
(:mod:`.hydro`), the batched ensemble (:mod:`.batch`) and the serving loop
(:mod:`.serve`).
"""
from ._abi import HydroParams, OCT_DTYPE  # noqa: F401

__version__ = "0.1.0"
