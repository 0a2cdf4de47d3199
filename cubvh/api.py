"""The reference's Python surface (cubvh/api.py) over the `_cubvh` torch
extension of this repository: same classes, functions, arguments, dtype and
device coercions, prefix-shape handling and errors (an unknown signed
distance mode raises KeyError, fewer than 9 triangles AssertionError,
backend failures RuntimeError)."""

import importlib.machinery
import importlib.util
import os
import sysconfig

import numpy as np
import torch


def _load_backend():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_cubvh" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not os.path.exists(path):
        raise ImportError(path + " is not built (python cubvh/_build.py, or __graft_entry__.build())")
    spec = importlib.util.spec_from_file_location("_cubvh", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_backend = _load_backend()

_sdf_mode_to_id = {
    'watertight': 0,
    'raystab': 1,
}


class cuBVH():
    def __init__(self, vertices, triangles):
        # vertices: np.ndarray / torch.Tensor, [N, 3]
        # triangles: np.ndarray / torch.Tensor, [M, 3]
        if torch.is_tensor(vertices): vertices = vertices.detach().cpu().numpy()
        if torch.is_tensor(triangles): triangles = triangles.detach().cpu().numpy()
        assert triangles.shape[0] > 8, "BVH needs at least 8 triangles."
        self.impl = _backend.create_cuBVH(np.asarray(vertices), np.asarray(triangles))

    def state_dict(self):
        # return: dict of str -> torch.Tensor (CPU): 'nodes' int32 [n, 9],
        # 'triangles' int32 [F, 12] (the reference's records), 'version' int32 [1]
        return self.impl.state_dict()

    @staticmethod
    def from_state_dict(state_dict):
        # state_dict: dict of str -> torch.Tensor (a version given as a
        # plain int is accepted too)
        sd = dict(state_dict)
        if "version" in sd and not torch.is_tensor(sd["version"]):
            sd["version"] = torch.tensor([sd["version"]]) if isinstance(sd["version"], int) \
                else torch.tensor([-1])
        impl = _backend.from_state_dict(sd)
        obj = cuBVH.__new__(cuBVH)
        obj.impl = impl
        return obj

    def ray_trace(self, rays_o, rays_d):
        # rays_o, rays_d: torch.Tensor, float, [..., 3]
        # return: positions [..., 3] f32, face_id [...] i64 (-1 on a miss),
        # depth [...] f32 (1000 on a miss)
        rays_o = rays_o.float().contiguous()
        rays_d = rays_d.float().contiguous()
        if not rays_o.is_cuda: rays_o = rays_o.cuda()
        if not rays_d.is_cuda: rays_d = rays_d.cuda()
        prefix = rays_o.shape[:-1]
        rays_o = rays_o.view(-1, 3)
        rays_d = rays_d.view(-1, 3)
        N = rays_o.shape[0]
        positions = torch.empty(N, 3, dtype=torch.float32, device=rays_o.device)
        face_id = torch.empty(N, dtype=torch.int64, device=rays_o.device)
        depth = torch.empty(N, dtype=torch.float32, device=rays_o.device)
        self.impl.ray_trace(rays_o, rays_d, positions, face_id, depth)
        return positions.view(*prefix, 3), face_id.view(*prefix), depth.view(*prefix)

    def _distance(self, positions, return_uvw, mode):
        positions = positions.float().contiguous()
        if not positions.is_cuda: positions = positions.cuda()
        prefix = positions.shape[:-1]
        positions = positions.view(-1, 3)
        N = positions.shape[0]
        distances = torch.empty(N, dtype=torch.float32, device=positions.device)
        face_id = torch.empty(N, dtype=torch.int64, device=positions.device)
        uvw = torch.empty(N, 3, dtype=torch.float32, device=positions.device) if return_uvw else None
        if mode is None:
            self.impl.unsigned_distance(positions, distances, face_id, uvw)
        else:
            self.impl.signed_distance(positions, distances, face_id, uvw, mode)
        distances = distances.view(*prefix)
        face_id = face_id.view(*prefix)
        if uvw is not None:
            uvw = uvw.view(*prefix, 3)
        return distances, face_id, uvw

    def unsigned_distance(self, positions, return_uvw=False):
        # positions: torch.Tensor, float, [..., 3]
        return self._distance(positions, return_uvw, None)

    def signed_distance(self, positions, return_uvw=False, mode='watertight'):
        # positions: torch.Tensor, float, [..., 3]; inside is negative
        return self._distance(positions, return_uvw, _sdf_mode_to_id[mode])


def floodfill(grid):
    # grid: torch.Tensor, bool, [B, H, W, D] or [H, W, D]
    # return: torch.Tensor, int32, same shape: -1 for occupied voxels, else the
    # smallest linear index of the voxel's free component (not remapped)
    grid = grid.contiguous()
    if not grid.is_cuda: grid = grid.cuda()
    if grid.dim() == 3:
        return _backend.floodfill(grid.unsqueeze(0)).squeeze(0)
    return _backend.floodfill(grid)


def sparse_marching_cubes(coords, corners, iso, ensure_consistency=False):
    # coords: torch.Tensor, int, [N, 3]; corners: torch.Tensor, float, [N, 8]
    # return: vertices float32 [M, 3], triangles int32 [T, 3] (CUDA)
    coords = coords.int().contiguous()
    corners = corners.float().contiguous()
    if not coords.is_cuda: coords = coords.cuda()
    corners = corners.to(coords.device)
    return _backend.sparse_marching_cubes(coords, corners, iso, ensure_consistency)
