"""nebula_b200: B200-native electron transport behind Nebula's interfaces.

The compute path is the CUDA library ``libnebula_b200.so`` (C ABI in
include/nebula_b200.h); this package is its Python host binding plus the
synthetic input generators used by the tests and the benchmark.
"""
from .api import (Geometry, Material, Simulation, Batch, PRI_DTYPE, TRI_DTYPE, DEPOSIT_DTYPE,  # noqa: F401
                  triangles_from_vertices, debug_events, physics_options, page_lock, page_unlock)
from ._capi import NblError, lib  # noqa: F401

__all__ = ["Geometry", "Material", "Simulation", "Batch", "PRI_DTYPE", "TRI_DTYPE", "DEPOSIT_DTYPE", "triangles_from_vertices",
           "debug_events", "physics_options", "page_lock", "page_unlock", "NblError", "lib"]
