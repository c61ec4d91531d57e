"""Seeded synthetic scenes and cameras for the LBVH build / closest-hit workloads.

The reference ships no data sets; its meshes come from an external model
library. These generators produce the host-side inputs that both the CUDA path
and the CPU oracle consume: float32 vertices as float4 (w = 0, the layout of
``CUDAMesh`` vertices, CUDAMesh.h) and uint32 faces as uint4 (a, b, c,
material), the layout of ``CUDAMesh`` faces. All randomness comes from numpy's
PCG64 generator seeded explicitly, so a (generator, seed) pair always yields
the same bytes on any host.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    vertices: np.ndarray  # (V, 4) float32, w = 0
    faces: np.ndarray  # (N, 4) uint32, (a, b, c, material)

    @property
    def face_count(self) -> int:
        return int(self.faces.shape[0])

    @property
    def vertex_count(self) -> int:
        return int(self.vertices.shape[0])

    def hitbox(self) -> np.ndarray:
        """min/max over every vertex, float4 each (CUDAModel grows its box per vertex)."""
        v = self.vertices
        return np.concatenate([v.min(axis=0), v.max(axis=0)]).astype(np.float32)


@dataclass
class Camera:
    center: tuple  # (x, y, z)
    target: tuple  # lookAt point
    fov: float  # radians, vertical (CUDA_calcPrimaryRays uses tan(fov/2) for up)
    width: int
    height: int

    @property
    def ratio(self) -> float:
        return float(np.float32(self.width) / np.float32(self.height))


def terrain(grid: int = 128, seed: int = 0, amplitude: float = 0.1, offset=(0.0, 0.0, 0.0), scale=(1.0, 1.0)) -> Mesh:
    """Height field on a grid x grid vertex lattice over x, z in [-1, 1].

    y = amplitude * sum_{k<4} sin(f_k * (cos(theta_k) x + sin(theta_k) z) + phi_k) with
    f_k ~ U[1, 8], phi_k ~ U[0, 2 pi), theta_k ~ U[0, 2 pi). Two triangles per
    cell: 2 (grid - 1)^2 faces (32,258 for grid = 128).
    """
    rng = np.random.default_rng(seed)
    f = rng.uniform(1.0, 8.0, 4)
    phi = rng.uniform(0.0, 2.0 * math.pi, 4)
    theta = rng.uniform(0.0, 2.0 * math.pi, 4)
    xs = np.linspace(-1.0, 1.0, grid)
    X, Z = np.meshgrid(xs, xs)  # rows: z, columns: x
    Y = np.zeros_like(X)
    for k in range(4):
        Y += np.sin(f[k] * (math.cos(theta[k]) * X + math.sin(theta[k]) * Z) + phi[k])
    Y *= amplitude
    verts = np.zeros((grid * grid, 4), dtype=np.float32)
    verts[:, 0] = (X.ravel() * scale[0] + offset[0]).astype(np.float32)
    verts[:, 1] = (Y.ravel() + offset[1]).astype(np.float32)
    verts[:, 2] = (Z.ravel() * scale[1] + offset[2]).astype(np.float32)
    i, j = np.meshgrid(np.arange(grid - 1), np.arange(grid - 1), indexing="ij")
    v00 = (i * grid + j).ravel()
    v01 = v00 + 1
    v10 = v00 + grid
    v11 = v10 + 1
    faces = np.zeros((2 * v00.size, 4), dtype=np.uint32)
    faces[0::2, 0], faces[0::2, 1], faces[0::2, 2] = v00, v10, v01
    faces[1::2, 0], faces[1::2, 1], faces[1::2, 2] = v01, v10, v11
    return Mesh(verts, faces)


def soup(n: int, seed: int = 1, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), sigma: float = 0.01) -> Mesh:
    """Triangle soup: centroids uniform in the box [lo, hi], each vertex = centroid + N(0, sigma^2) per axis."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(lo, hi, (n, 3))
    v = c[:, None, :] + rng.normal(0.0, sigma, (n, 3, 3))
    verts = np.zeros((3 * n, 4), dtype=np.float32)
    verts[:, :3] = v.reshape(3 * n, 3).astype(np.float32)
    faces = np.zeros((n, 4), dtype=np.uint32)
    faces[:, 0] = np.arange(0, 3 * n, 3, dtype=np.uint32)
    faces[:, 1] = faces[:, 0] + 1
    faces[:, 2] = faces[:, 0] + 2
    return Mesh(verts, faces)


def concat(*meshes: Mesh) -> Mesh:
    verts, faces, base = [], [], 0
    for m in meshes:
        verts.append(m.vertices)
        f = m.faces.copy()
        f[:, :3] += np.uint32(base)
        faces.append(f)
        base += m.vertex_count
    return Mesh(np.concatenate(verts), np.concatenate(faces))


# ----------------------------------------------------------------------------
# Workloads
# ----------------------------------------------------------------------------
FOV_60 = float(np.float32(math.pi / 3.0))


def terrain_small_scene(width: int = 512, height: int = 512, seed: int = 0):
    """Height-field terrain, 128 x 128 vertices (32,258 triangles); 512 x 512
    pinhole rays, 60 degree field of view, camera (0, 1.5, -2.5) looking at the origin."""
    return terrain(128, seed), Camera((0.0, 1.5, -2.5), (0.0, 0.0, 0.0), FOV_60, width, height)


def soup_1m_scene(width: int = 1920, height: int = 1080, seed: int = 1, n: int = 1 << 20):
    """Incoherent single scene: 2^20-triangle soup in the unit cube (vertex noise
    sigma 0.01); 1920 x 1080 primary rays from (0.5, 0.5, -0.4) looking at the
    cube's centre, so that the cube fills the frame, plus one diffuse bounce per hit."""
    return soup(n, seed), Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), FOV_60, width, height)


def batch_meshes(count: int = 1024, seed: int = 3, min_faces: int = 64, max_faces: int = 65536):
    """Independent meshes with face counts log-uniform in [min_faces, max_faces],
    each a terrain (side chosen so that 2 (s-1)^2 is near the count) or a soup
    by a fair coin. Returns the list of meshes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(min_faces), math.log(max_faces)))))
        if rng.random() < 0.5:
            side = max(2, int(round(math.sqrt(n / 2.0))) + 1)
            out.append(terrain(side, seed=int(rng.integers(1 << 30))))
        else:
            out.append(soup(n, seed=int(rng.integers(1 << 30))))
    return out


def concat_batch(meshes):
    """Concatenation for the batched build: faces keep indices local to their mesh."""
    fo, vo = [0], [0]
    for m in meshes:
        fo.append(fo[-1] + m.face_count)
        vo.append(vo[-1] + m.vertex_count)
    verts = np.concatenate([m.vertices for m in meshes])
    faces = np.concatenate([m.faces for m in meshes])
    return verts, faces, fo, vo


def learned_scene(scale: float = 1.0, seed: int = 4):
    """Terrain + soup for the learned proposal: a 512 x 512 height field (522,242
    triangles) with 3,500,000 soup triangles (vertex noise sigma 0.01) whose
    centroids are uniform in the 2 x 0.5 x 2 box x, z in [-1, 1], y in [0.45, 0.95]
    above it (the terrain spans y in [-0.4, 0.4]). `scale` shrinks both triangle
    counts (grid side ~ 512 sqrt(scale)) for smaller test cases."""
    side = max(8, int(round(511 * math.sqrt(scale)))) + 1
    t = terrain(side, seed)
    s = soup(max(1, int(round(3_500_000 * scale))), seed + 1, lo=(-1.0, 0.45, -1.0), hi=(1.0, 0.95, 1.0))
    return concat(t, s)


def instance_cameras(count: int, width: int, height: int, radius: float = 2.4, y: float = 1.3, target=(0.0, 0.2, 0.0)):
    """One pinhole camera per instance of the instanced learned scene, on a
    ring of `radius` around the scene at height y, each looking at `target`."""
    cams = []
    for i in range(count):
        a = 2.0 * math.pi * (i + 0.5) / count
        cams.append(Camera((radius * math.cos(a), y, radius * math.sin(a)), tuple(target), FOV_60, width, height))
    return cams


def displace_instances(base_vertices, count: int, frame: int, seed: int = 7, sigma: float = 0.002, out=None):
    """`count` copies of a device vertex array (float4), each vertex moved by
    N(0, sigma^2) per axis, drawn on the device from a generator seeded by
    (seed, frame): instance i is rows i V .. (i + 1) V of the result."""
    import torch

    V = base_vertices.shape[0]
    dev = base_vertices.device
    g = torch.Generator(device=dev).manual_seed(seed * 1_000_003 + frame)
    if out is None:
        out = torch.empty((count * V, 4), dtype=torch.float32, device=dev)
    out.view(count, V, 4).copy_(base_vertices.unsqueeze(0).expand(count, V, 4))
    out[:, :3] += sigma * torch.randn((count * V, 3), generator=g, device=dev)
    return out


def scene_box(mesh: Mesh, factor: float = 1.5):
    """The mesh's bounding box grown by `factor` about its centre (lo xyz, hi xyz)."""
    v = mesh.vertices[:, :3].astype(np.float64)
    lo, hi = v.min(0), v.max(0)
    c, h = 0.5 * (lo + hi), 0.5 * (hi - lo) * factor
    return tuple(float(x) for x in np.concatenate([c - h, c + h]))


def box_rays_torch(count: int, box, seed: int, device="cuda"):
    """`count` rays with origins uniform in `box` and directions uniform on the
    unit sphere (float4, w = 0), drawn on the device from a seeded generator."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    lo = torch.tensor(box[:3], dtype=torch.float32, device=device)
    hi = torch.tensor(box[3:], dtype=torch.float32, device=device)
    o = torch.zeros((count, 4), dtype=torch.float32, device=device)
    d = torch.zeros((count, 4), dtype=torch.float32, device=device)
    o[:, :3] = lo + (hi - lo) * torch.rand((count, 3), generator=g, device=device)
    v = torch.randn((count, 3), generator=g, device=device)
    d[:, :3] = v / v.norm(dim=1, keepdim=True).clamp(min=1e-30)
    return o, d


def sphere_rays(mesh: Mesh, side: int, seed: int):
    """side x side rays with origins uniform on the mesh's bounding sphere, each
    aimed at a uniform point inside the sphere (float32 float4 origin, direction)."""
    rng = np.random.default_rng(seed)
    v = mesh.vertices[:, :3].astype(np.float64)
    c = 0.5 * (v.min(0) + v.max(0))
    r = max(float(np.linalg.norm(v - c, axis=1).max()), 1e-6) * 1.01
    R = side * side
    p = rng.normal(size=(R, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    q = rng.normal(size=(R, 3))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q *= rng.uniform(size=(R, 1)) ** (1.0 / 3.0)
    o = c + r * p
    d = (c + r * q) - o
    orig = np.zeros((R, 4), np.float32)
    dirs = np.zeros((R, 4), np.float32)
    orig[:, :3] = o
    dirs[:, :3] = d
    return orig, dirs


def batch_sphere_rays_torch(meshes, seed_sides: int = 11, seed_rays: int = 5, min_side: int = 64, max_side: int = 512,
                            device="cuda"):
    """Ray sets of a batch of meshes: mesh m gets side x side rays (side log-uniform in [min_side, max_side],
    numpy PCG64 seeded by seed_sides) with origins uniform on its bounding sphere (centre of its vertex box,
    radius 1.01 x the farthest vertex), each aimed at a uniform point inside that sphere; drawn in float64 on
    the device from a generator seeded by seed_rays. Returns (orig, dir, ray_offsets) with ray_offsets an
    int64 numpy array of mesh_count + 1 entries."""
    import torch

    count = len(meshes)
    rng = np.random.default_rng(seed_sides)
    sides = np.exp(rng.uniform(math.log(min_side), math.log(max_side), count)).astype(np.int64)
    counts = sides * sides
    ro = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    centers, radii = [], []
    for m in meshes:
        v = m.vertices[:, :3].astype(np.float64)
        c = 0.5 * (v.min(0) + v.max(0))
        centers.append(c)
        radii.append(max(float(np.linalg.norm(v - c, axis=1).max()), 1e-6) * 1.01)
    R = int(ro[-1])
    mesh_of_ray = torch.repeat_interleave(torch.arange(count, device=device), torch.from_numpy(counts).to(device))
    cen = torch.tensor(np.array(centers), dtype=torch.float64, device=device)[mesh_of_ray]
    rad = torch.tensor(radii, dtype=torch.float64, device=device)[mesh_of_ray].unsqueeze(1)
    g = torch.Generator(device=device).manual_seed(seed_rays)
    p = torch.randn((R, 3), generator=g, device=device, dtype=torch.float64)
    p = p / p.norm(dim=1, keepdim=True)
    q = torch.randn((R, 3), generator=g, device=device, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True) * torch.rand((R, 1), generator=g, device=device, dtype=torch.float64).pow(1.0 / 3.0)
    orig = torch.zeros((R, 4), dtype=torch.float32, device=device)
    dirs = torch.zeros((R, 4), dtype=torch.float32, device=device)
    orig[:, :3] = (cen + rad * p).float()
    dirs[:, :3] = ((cen + rad * q) - (cen + rad * p)).float()
    return orig, dirs, ro
