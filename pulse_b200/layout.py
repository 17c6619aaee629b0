"""Device data layout of the scene: the 13 storage buffers of pulse's scene bind group.

The byte layout is the std430 layout of the WGSL structs in
``src/scene/types.wgsl:3-74`` as written by encase from the Rust structs in
``src/scene/mod.rs`` (``PulsePrimitive`` :344, ``PulseTriangleData`` :338,
``PulseBLASNode`` ``src/scene/blas.rs:5``, ``PulseTLASNode`` ``src/scene/tlas.rs:4``,
``PulseMeshInstance`` :527, ``PulseMaterial`` :240, ``PulseLightDataIndex`` :547).
Every array here is a plain numpy array whose rows are those structs viewed as
32-bit words, so the same buffers feed the CUDA library's raw upload entry point
and the CPU oracle.

``triangle_soup`` restates the per-mesh triangle-soup extraction of
``prepare_extracted_mesh_assets`` (``src/scene/mod.rs:410-424``); it only copies
vertex attributes through the index buffer, no arithmetic.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

PRIM_WORDS = 12      # 48 B: vec3 p0 @0, p1 @16, p2 @32
TRIDATA_WORDS = 20   # 80 B: vec3 n0 @0, n1 @16, n2 @32, vec2 uv0 @48, uv1 @56, uv2 @64
NODE_WORDS = 8       # 32 B: vec3 min, u32 a_or_first, vec3 max, u32 count
INSTANCE_WORDS = 40  # 160 B: mat4 object_world, mat4 world_object, 5 x u32, pad
MATERIAL_WORDS = 12  # 48 B: vec4 base_color, vec4 emissive, roughness, reflectance, metallic, pad

# Offsets of the u32 fields of a MeshInstance row (in 32-bit words).
INST_TRIANGLE_OFFSET = 32
INST_TRIANGLE_COUNT = 33
INST_INDEX_OFFSET = 34
INST_NODE_OFFSET = 35
INST_MATERIAL_INDEX = 36


@dataclass
class Mesh:
    """An indexed triangle mesh with the three attributes pulse extracts
    (POSITION f32x3, NORMAL f32x3, UV_0 f32x2; ``src/scene/mod.rs:376-400``)."""

    positions: np.ndarray   # (V, 3) f32
    normals: np.ndarray     # (V, 3) f32
    uvs: np.ndarray         # (V, 2) f32
    indices: np.ndarray     # (3T,) u32

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float32)
        self.normals = np.ascontiguousarray(self.normals, dtype=np.float32)
        self.uvs = np.ascontiguousarray(self.uvs, dtype=np.float32)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.uint32).reshape(-1)

    @property
    def triangle_count(self) -> int:
        return self.indices.size // 3


@dataclass
class Material:
    """The StandardMaterial subset pulse reads (``src/scene/mod.rs:255-262``)."""

    base_color: tuple = (1.0, 1.0, 1.0, 1.0)
    emissive: tuple = (0.0, 0.0, 0.0, 1.0)
    perceptual_roughness: float = 0.5
    reflectance: float = 0.5
    metallic: float = 0.0

    def to_words(self) -> np.ndarray:
        row = np.zeros(MATERIAL_WORDS, dtype=np.float32)
        bc = list(self.base_color) + [1.0] * (4 - len(self.base_color))
        em = list(self.emissive) + [1.0] * (4 - len(self.emissive))
        row[0:4] = bc[:4]
        row[4:8] = em[:4]
        row[8] = self.perceptual_roughness
        row[9] = self.reflectance
        row[10] = self.metallic
        return row


@dataclass
class Instance:
    """One (mesh, material, GlobalTransform) triple (``src/scene/mod.rs:517-525``).
    ``object_world`` is a 4x4 row-major numpy matrix (it is stored column-major)."""

    mesh: int
    material: int
    object_world: np.ndarray = field(default_factory=lambda: np.eye(4))

    def columns(self) -> np.ndarray:
        return np.ascontiguousarray(np.asarray(self.object_world, dtype=np.float32).T).reshape(16)


def triangle_soup(mesh: Mesh):
    """(primitives (T,12) f32, triangle_data (T,20) f32) in std430 rows."""
    idx = mesh.indices.reshape(-1, 3)
    t = idx.shape[0]
    prims = np.zeros((t, PRIM_WORDS), dtype=np.float32)
    tdata = np.zeros((t, TRIDATA_WORDS), dtype=np.float32)
    for k in range(3):
        prims[:, 4 * k:4 * k + 3] = mesh.positions[idx[:, k]]
        tdata[:, 4 * k:4 * k + 3] = mesh.normals[idx[:, k]]
        tdata[:, 12 + 2 * k:14 + 2 * k] = mesh.uvs[idx[:, k]]
    return prims, tdata


@dataclass
class SceneBuffers:
    """The 13 buffers of the scene bind group plus the uniform
    (``src/scene/bindings.wgsl:14-28``).  Word arrays, C-contiguous."""

    instance_count: int
    light_count: int
    primitives: np.ndarray                   # (T, 12) f32
    triangle_data: np.ndarray                # (T, 20) f32
    triangle_indices: np.ndarray             # (T,) u32
    blas_nodes: np.ndarray                   # (N, 8) u32
    tlas_nodes: np.ndarray                   # (M, 8) u32
    instance_indices: np.ndarray             # (K,) u32
    instances: np.ndarray                    # (K, 40) u32
    materials: np.ndarray                    # (Mt, 12) f32
    light_emission_strength_cdf: np.ndarray  # (L,) f32
    light_triangle_area_cdfs: np.ndarray     # (C,) f32
    light_mesh_areas: np.ndarray             # (L,) f32
    light_indices: np.ndarray                # (L, 2) u32
    # per-mesh {triangle_offset, triangle_count, index_offset, node_offset}
    mesh_index: np.ndarray = None            # (Meshes, 4) u32

    def arrays(self):
        return [self.primitives, self.triangle_data, self.triangle_indices, self.blas_nodes,
                self.tlas_nodes, self.instance_indices, self.instances, self.materials,
                self.light_emission_strength_cdf, self.light_triangle_area_cdfs,
                self.light_mesh_areas, self.light_indices]


def node_fields(nodes: np.ndarray):
    """Split a (N, 8) u32 node array into (min (N,3) f32, a (N,), max (N,3) f32, count (N,))."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    mn = nodes[:, 0:3].view(np.float32)
    mx = nodes[:, 4:7].view(np.float32)
    return mn, nodes[:, 3], mx, nodes[:, 7]


def empty_f32(n, w=None):
    return np.zeros((n, w) if w else (n,), dtype=np.float32)


def empty_u32(n, w=None):
    return np.zeros((n, w) if w else (n,), dtype=np.uint32)
