"""cubvh_b200: B200-native (sm_100a) mesh queries behind cubvh's Python API.

    import cubvh_b200 as cubvh
    bvh = cubvh.cuBVH(vertices, faces)
    dist, face_id, uvw = bvh.unsigned_distance(points, return_uvw=True)
    sdf, face_id, _ = bvh.signed_distance(points, mode="watertight")
    pos, face_id, depth = bvh.ray_trace(rays_o, rays_d)
    labels = cubvh.floodfill(occupancy)
    sdf = cubvh.udf_to_sdf(udf_grid)     # occupancy -> floodfill -> signed grid, fused
"""

from ._lib import version
from .api import cuBVH, floodfill, sparse_marching_cubes, udf_to_sdf
from .arena import BVHArena

__all__ = ["cuBVH", "floodfill", "udf_to_sdf", "sparse_marching_cubes", "BVHArena", "version"]
