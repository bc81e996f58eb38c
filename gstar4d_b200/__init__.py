"""gStar4D-B200: B200-native (sm_100a) 3D Delaunay triangulation by star splaying.

Point cloud in, tetrahedra with adjacency out, bit-exact with the reference
gStar4D under its Simulation of Simplicity. The compute path is the CUDA
library libgstar4d.so behind the C ABI of include/gstar4d.h; this package is
its Python host mirror (api), the benchmark workloads, and the CLI.
"""
from .api import (G4DError, Triangulator, default_config, load, tets_as_array,  # noqa: F401
                  triangulate, TET_DTYPE)

__all__ = ["G4DError", "Triangulator", "default_config", "load", "tets_as_array", "triangulate", "TET_DTYPE"]
