"""vorothree_b200 -- B200-native 3D Voronoi tessellation.

A GPU drop-in for the reference crate ``voronoid``'s 3D path
(Tessellation::calculate over Algorithm3DGrid + Cell3DFaces, with plane,
sphere, cylinder, cone, torus and convex-polyhedron walls).  The work runs in hand-written sm_100a CUDA kernels behind a C
ABI (include/voronoid_b200.h); this package is the Python mirror of the
reference's API over that ABI.
"""
from ._lib import VoronoidError, load
from .batch import TessellationBatch
from .server import TessellationServer
from .shard import (calculate_sharded, calculate_sharded_device, calculate_sharded_faces,
                    calculate_sharded_faces_device, cell_chunks, cell_range, device_neighbors, device_summaries,
                    gather_cells_tensors, gather_summaries, gather_summaries_tensors, set_generators_broadcast)
from .tessellation import (WALL_ID_MAX, Algorithm3DGrid, BoundingBox, Cell3DFaces, ConeGeometry,
                           ConvexPolyhedronGeometry, CylinderGeometry, PlaneGeometry, SphereGeometry, Tessellation,
                           TorusGeometry, Wall, box_side, parse_generators)

__all__ = ["Algorithm3DGrid", "BoundingBox", "Cell3DFaces", "ConeGeometry", "ConvexPolyhedronGeometry",
           "CylinderGeometry", "PlaneGeometry", "SphereGeometry", "TorusGeometry",
           "Tessellation", "TessellationBatch", "TessellationServer", "Wall", "WALL_ID_MAX", "box_side", "VoronoidError", "load",
           "calculate_sharded", "calculate_sharded_device", "calculate_sharded_faces", "calculate_sharded_faces_device",
           "cell_chunks", "cell_range", "device_neighbors", "device_summaries", "gather_cells_tensors",
           "gather_summaries",
           "gather_summaries_tensors", "parse_generators", "set_generators_broadcast"]
