"""Drop-in for the reference's `cubvh` Python package (cubvh/__init__.py,
cubvh/api.py) on the hot path: cuBVH (unsigned_distance, signed_distance
in 'watertight' and 'raystab' modes, ray_trace, state_dict /
from_state_dict), floodfill and sparse_marching_cubes, with the reference's
names, arguments and return shapes.  Calls go through the `_cubvh` torch
extension (cubvh/csrc/bindings.cpp), a thin layer over the C ABI of
libcubvh_b200.so, whose CUDA kernels run the queries.

The reference's other exports (hash tables, hole filling, vertex merging,
decimation, CPU marching cubes) are not part of this library; asking for
them raises AttributeError.  Extras (autograd, batched arenas, the fused
udf_to_sdf, host-buffer queries) live in the cubvh_b200 package.
"""

from .api import cuBVH, floodfill, sparse_marching_cubes

__all__ = ["cuBVH", "floodfill", "sparse_marching_cubes"]

_NOT_HERE = ("HashTable", "cuHashTable", "sparse_marching_cubes_cpu", "fill_holes", "merge_vertices", "decimate",
             "parallel_decimate")


def __getattr__(name):
    if name in _NOT_HERE:
        raise AttributeError(f"cubvh.{name} is outside this library's scope (mesh queries and floodfill only)")
    raise AttributeError(f"module 'cubvh' has no attribute {name!r}")
