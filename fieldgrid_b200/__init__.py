"""B200-native Yee-grid FDTD engine with the API of v0l/fieldgrid's `sims_field::fdtd`.

Modules: `fdtd` (Sim, run, Extras, Pulse, Record, patches, Far), `grid` (Grid and node-line
helpers), `gpu` (Gpu). The engine itself is libfieldgrid.so (CUDA for sm_100a + C++ host
setup) behind the C ABI declared in include/fieldgrid.h.
"""
from .grid import Grid  # noqa: F401

__all__ = ["Grid", "fdtd", "grid", "gpu"]
