"""Seeded procedural scenes for the benchmark and parity workloads.

All inputs are synthetic (no datasets): the Cornell box, displaced icospheres,
an fBm terrain with instanced rocks, and the mixed batch of scenes.  Geometry
is generated in float64 with numpy and rounded once to float32, so the same
seed gives the same bytes on every machine with this numpy.

The camera follows Bevy 0.13's defaults, which is what pulse's demo uses
(``src/main.rs:105-125``): ``PerspectiveProjection{fov: pi/4, near: 0.1}``
through ``Mat4::perspective_infinite_reverse_rh``; the shader receives
``view.inverse_view_proj`` and ``view.world_position``
(``src/path_tracer/path_tracer.wgsl:69-73``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .layout import Instance, Material, Mesh


# ----------------------------------------------------------------- camera --
@dataclass
class View:
    inverse_view_proj: np.ndarray  # (16,) f32, column-major
    world_position: np.ndarray     # (3,) f32


def _look_rotation(eye, target, up=(0.0, 1.0, 0.0)):
    eye, target, up = (np.asarray(v, dtype=np.float64) for v in (eye, target, up))
    back = eye - target
    back /= np.linalg.norm(back)
    right = np.cross(up, back)
    right /= np.linalg.norm(right)
    up2 = np.cross(back, right)
    return np.stack([right, up2, back], axis=1)  # columns: local x, y, z


def bevy_view(eye, target=None, aspect=1.0, fov_y=math.pi / 4, near=0.1) -> View:
    """inverse(projection * view) for a Bevy camera at ``eye`` looking at ``target``
    (default: down -Z), projection = perspective_infinite_reverse_rh."""
    eye = np.asarray(eye, dtype=np.float64)
    rot = np.eye(3) if target is None else _look_rotation(eye, target)
    cam = np.eye(4)
    cam[:3, :3] = rot
    cam[:3, 3] = eye
    f = 1.0 / math.tan(0.5 * fov_y)
    proj = np.zeros((4, 4))
    proj[0, 0] = f / aspect
    proj[1, 1] = f
    proj[3, 2] = -1.0
    proj[2, 3] = near
    inv_vp = cam @ np.linalg.inv(proj)
    return View(np.ascontiguousarray(inv_vp.T.astype(np.float32)).reshape(16),
                eye.astype(np.float32))


# ------------------------------------------------------------- transforms --
def trs(translation=(0, 0, 0), rotation=None, scale=(1, 1, 1)) -> np.ndarray:
    m = np.eye(4)
    r = np.eye(3) if rotation is None else np.asarray(rotation, dtype=np.float64)
    m[:3, :3] = r @ np.diag(np.asarray(scale, dtype=np.float64) * np.ones(3))
    m[:3, 3] = translation
    return m


def rot_y(angle):
    c, s = math.cos(angle), math.sin(angle)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
    ])


# ----------------------------------------------------------------- meshes --
def quad_mesh(corners, normal) -> Mesh:
    """Two triangles (0,1,2), (0,2,3) over four corners, flat normal."""
    p = np.asarray(corners, dtype=np.float64)
    n = np.tile(np.asarray(normal, dtype=np.float64), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
    return Mesh(p, n, uv, np.array([0, 1, 2, 0, 2, 3], dtype=np.uint32))


def unit_cube() -> Mesh:
    """Axis-aligned cube [-0.5, 0.5]^3, 12 triangles, outward flat normals."""
    pos, nrm, uv, idx = [], [], [], []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = sgn
            u = np.zeros(3)
            u[(axis + 1) % 3] = 1.0
            v = np.cross(n, u)
            c = 0.5 * n
            base = len(pos)
            for a, b in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                pos.append(c + 0.5 * a * u + 0.5 * b * v)
                nrm.append(n)
                uv.append(((a + 1) / 2, (b + 1) / 2))
            idx += [base, base + 1, base + 2, base, base + 2, base + 3]
    return Mesh(np.array(pos), np.array(nrm), np.array(uv), np.array(idx, dtype=np.uint32))


def disc_mesh(n_tris: int, radius: float = 1.0) -> Mesh:
    """Flat triangle fan in the xz plane facing -y (a downward emitter)."""
    ang = np.arange(n_tris) * (2 * math.pi / n_tris)
    rim = np.stack([radius * np.cos(ang), np.zeros(n_tris), radius * np.sin(ang)], axis=1)
    pos = np.vstack([np.zeros((1, 3)), rim])
    nrm = np.tile([0.0, -1.0, 0.0], (n_tris + 1, 1))
    uv = np.vstack([[0.5, 0.5], 0.5 + 0.5 * rim[:, [0, 2]] / radius])
    tri = np.stack([np.zeros(n_tris, dtype=np.int64), 1 + (np.arange(n_tris) + 1) % n_tris,
                    1 + np.arange(n_tris)], axis=1)
    return Mesh(pos, nrm, uv, tri.reshape(-1).astype(np.uint32))


def icosphere(level: int):
    """Unit icosphere (vertices float64 (V,3), faces int64 (20*4^level, 3))."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        nv = v.shape[0]
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        e = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        key = np.sort(e, axis=1)
        uniq, inv = np.unique(key[:, 0] * nv + key[:, 1], return_inverse=True)
        ua, ub = uniq // nv, uniq % nv
        mid = v[ua] + v[ub]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.vstack([v, mid])
        m = (nv + inv).reshape(-1, 3)
        mab, mbc, mca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, mab, mca], 1), np.stack([b, mbc, mab], 1),
                            np.stack([c, mca, mbc], 1), np.stack([mab, mbc, mca], 1)])
    return v, f


class ValueNoise:
    """Seeded 3-D value noise in [-1, 1] (hashed lattice values, smoothstep
    trilinear interpolation)."""

    def __init__(self, seed: int):
        rng = np.random.default_rng(seed)
        self.perm = rng.permutation(256).astype(np.int64)
        self.vals = rng.uniform(-1.0, 1.0, 256)

    def _h(self, ix, iy, iz):
        p = self.perm
        return self.vals[p[(p[(p[ix & 255] + iy) & 255] + iz) & 255]]

    def __call__(self, pts):
        pts = np.asarray(pts, dtype=np.float64)
        i = np.floor(pts).astype(np.int64)
        fr = pts - i
        u = fr * fr * (3.0 - 2.0 * fr)
        out = np.zeros(pts.shape[0])
        for dx in (0, 1):
            wx = u[:, 0] if dx else 1.0 - u[:, 0]
            for dy in (0, 1):
                wy = u[:, 1] if dy else 1.0 - u[:, 1]
                for dz in (0, 1):
                    wz = u[:, 2] if dz else 1.0 - u[:, 2]
                    out += wx * wy * wz * self._h(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        return out

    def grid(self, xs, ys, z: float):
        """self(pts) for the points (xs[j], ys[i], z) of a grid, as an
        (len(ys), len(xs)) array, bit for bit: the lattice hashes and weights
        of a row or column are computed once, the per-point products and the
        sum run in the same order as __call__."""
        xs = np.asarray(xs, dtype=np.float64)
        ys = np.asarray(ys, dtype=np.float64)
        ix = np.floor(xs).astype(np.int64)
        iy = np.floor(ys).astype(np.int64)
        iz = int(np.floor(z))
        ux, uy = xs - ix, ys - iy
        ux = ux * ux * (3.0 - 2.0 * ux)
        uy = uy * uy * (3.0 - 2.0 * uy)
        fz = z - iz
        uz = fz * fz * (3.0 - 2.0 * fz)
        # hashes over the distinct lattice columns / rows only
        cx, jx = np.unique(ix, return_inverse=True)
        cy, jy = np.unique(iy, return_inverse=True)
        out = np.zeros((ys.size, xs.size))
        wxy = np.empty_like(out)
        term = np.empty_like(out)
        for dx in (0, 1):
            wx = ux if dx else 1.0 - ux
            for dy in (0, 1):
                wy = uy if dy else 1.0 - uy
                np.multiply(wx[None, :], wy[:, None], out=wxy)
                for dz in (0, 1):
                    wz = uz if dz else 1.0 - uz
                    h = self._h(cx[None, :] + dx, cy[:, None] + dy, np.int64(iz + dz))
                    np.multiply(wxy, wz, out=term)
                    term *= h[np.ix_(jy, jx)]
                    out += term
        return out


def vertex_normals(v, f):
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    # np.add.at(n, f[:, k], fn) for k = 0, 1, 2 in turn, as one bincount per
    # component over the three index columns in that order (the same sequence
    # of float64 additions per vertex, much faster)
    idx = f.T.reshape(-1)
    n = np.stack([np.bincount(idx, weights=np.tile(fn[:, c], 3), minlength=v.shape[0]) for c in range(3)], 1)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    ln[ln == 0] = 1.0
    return n / ln


def displaced_icosphere(level: int, amplitude: float = 0.1, seed: int = 0, freq: float = 3.0,
                        radius: float = 1.0) -> Mesh:
    """Icosphere of 20*4^level triangles, radius * (1 + amplitude * noise(freq * p))."""
    v, f = icosphere(level)
    noise = ValueNoise(seed)
    r = radius * (1.0 + amplitude * noise(v * freq))
    v = v * r[:, None]
    n = vertex_normals(v, f)
    uv = np.stack([0.5 + np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi),
                   0.5 - np.arcsin(np.clip(v[:, 1] / np.linalg.norm(v, axis=1), -1, 1)) / math.pi], 1)
    return Mesh(v, n, uv, f.reshape(-1).astype(np.uint32))


def fbm_grid(n: int, size: float, height: float, seed: int, octaves: int = 6) -> Mesh:
    """n x n vertex heightfield over [-size/2, size/2]^2, 2*(n-1)^2 triangles."""
    noise = ValueNoise(seed)
    xs = np.linspace(-size / 2, size / 2, n)
    gx, gz = np.meshgrid(xs, xs, indexing="xy")
    pts = np.stack([gx.ravel(), np.zeros(n * n), gz.ravel()], 1)
    h = np.zeros(n * n)
    amp, fr = 1.0, 4.0 / size
    for _ in range(octaves):
        # noise at (x * fr, z * fr, 0.37 * fr * size) of every grid point
        h += amp * noise.grid(xs * fr, xs * fr, 0.37 * fr * size).reshape(-1)
        amp *= 0.5
        fr *= 2.0
    pts[:, 1] = height * h
    ij = np.arange(n * n).reshape(n, n)
    a = ij[:-1, :-1].ravel()
    b = ij[:-1, 1:].ravel()
    c = ij[1:, 1:].ravel()
    d = ij[1:, :-1].ravel()
    f = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b], 1)])
    nrm = vertex_normals(pts, f)
    uv = np.stack([(gx.ravel() / size) + 0.5, (gz.ravel() / size) + 0.5], 1)
    return Mesh(pts, nrm, uv, f.reshape(-1).astype(np.uint32))


# ----------------------------------------------------------------- scenes --
# Mesh scale and the reference's ray/triangle epsilon.  pulse rejects a
# triangle as parallel when |e1 . (d x e2)| < 1e-4 in object space
# (src/utilities.wgsl:437), an absolute threshold: a triangle of edge length e
# is only visible where |cos(incidence)| > ~1.15e-4 / e^2.  A unit icosphere at
# subdivision 7 has e ~ 0.008 and is invisible at every angle, so the sphere
# meshes here are generated large enough in object space (edge >= ~0.02) for
# the reference's constants to render them.

def sphere_radius_for(level: int, min_edge: float = 0.02) -> float:
    """Object-space radius giving icosphere edges of at least min_edge."""
    return max(1.0, min_edge * (2 ** level) / 1.0515)

@dataclass
class SceneDesc:
    name: str
    meshes: list
    materials: list
    instances: list
    view: View
    width: int
    height: int
    params: dict = field(default_factory=dict)

    @property
    def triangle_count(self) -> int:
        return sum(self.meshes[i.mesh].triangle_count for i in self.instances)


def cornell(width: int = 256, height: int = 256) -> SceneDesc:
    """Cornell box of 36 triangles: 5 wall quads, 2 rotated boxes (a unit cube
    mesh instanced twice, +/-18 degrees about y) and a ceiling light quad of
    radiance (17, 12, 4)."""
    white = Material((0.73, 0.73, 0.73, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0)
    red = Material((0.65, 0.05, 0.05, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0)
    green = Material((0.12, 0.45, 0.15, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0)
    light = Material((0.78, 0.78, 0.78, 1), (17.0, 12.0, 4.0, 1), 1.0, 0.5, 0.0)
    meshes = [
        quad_mesh([(-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)], (0, 1, 0)),     # floor
        quad_mesh([(-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)], (0, -1, 0)),        # ceiling
        quad_mesh([(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)], (0, 0, 1)),     # back
        quad_mesh([(-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1)], (1, 0, 0)),     # left
        quad_mesh([(1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)], (-1, 0, 0)),        # right
        unit_cube(),
        quad_mesh([(-0.25, 0.98, -0.25), (0.25, 0.98, -0.25), (0.25, 0.98, 0.25), (-0.25, 0.98, 0.25)],
                  (0, -1, 0)),                                                           # light
    ]
    materials = [white, red, green, light, Material((0.73, 0.73, 0.73, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0),
                 Material((0.73, 0.73, 0.73, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0),
                 Material((0.73, 0.73, 0.73, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0),
                 Material((0.73, 0.73, 0.73, 1), (0, 0, 0, 1), 1.0, 0.5, 0.0)]
    instances = [
        Instance(0, 0), Instance(1, 4), Instance(2, 5), Instance(3, 1), Instance(4, 2),
        Instance(5, 6, trs((-0.33, -0.4, -0.3), rot_y(math.radians(18.0)), (0.55, 1.2, 0.55))),
        Instance(5, 7, trs((0.35, -0.7, 0.3), rot_y(math.radians(-18.0)), (0.6, 0.6, 0.6))),
        Instance(6, 3),
    ]
    view = bevy_view((0.0, 0.0, 3.0), None, aspect=width / height)
    return SceneDesc("cornell", meshes, materials, instances, view, width, height,
                     dict(max_depth=4, nee_mode=2, light_pick=1, bins=16, max_leaf=4))


def spheres_1080p(seed: int = 0, level: int = 7, n_instances: int = 64, n_light_patches: int = 8,
                  tris_per_patch: int = 32, width: int = 1920, height: int = 1080, box: float = 10.0) -> SceneDesc:
    """64 rigid instances of one displaced icosphere (subdivision 7, 327,680
    triangles, noise amplitude 0.1, object-space radius from sphere_radius_for:
    2.43 at subdivision 7) placed in a 20^3 box; per-instance GGX roughness
    U(0.05, 1), metallic Bernoulli(0.3), albedo U(0, 1)^3; 8 emissive patches of
    32 triangles (256 emissive triangles) of radiance U(1, 20) above the box."""
    rng = np.random.default_rng(seed)
    radius = sphere_radius_for(level)
    sphere = displaced_icosphere(level, 0.1, seed, radius=radius)
    patch = disc_mesh(tris_per_patch, 1.5)
    meshes = [sphere, patch]
    materials, instances = [], []
    for i in range(n_instances):
        rough = rng.uniform(0.05, 1.0)
        metal = float(rng.random() < 0.3)
        albedo = rng.uniform(0.0, 1.0, 3)
        materials.append(Material((*albedo, 1.0), (0, 0, 0, 1), rough, 0.5, metal))
        instances.append(Instance(0, i, trs(rng.uniform(-box, box, 3), random_rotation(rng))))
    for j in range(n_light_patches):
        le = rng.uniform(1.0, 20.0)
        materials.append(Material((0.8, 0.8, 0.8, 1), (le, le, le, 1), 1.0, 0.5, 0.0))
        gx, gz = (j % 4) - 1.5, (j // 4) - 0.5
        instances.append(Instance(1, n_instances + j, trs((gx * 5.0, 10.0 + 1.5 * radius, gz * 8.0))))
    view = bevy_view((0.0, 2.0, 18.0 + 3.0 * radius), (0.0, 0.0, 0.0), aspect=width / height)
    return SceneDesc("spheres_1080p", meshes, materials, instances, view, width, height,
                     dict(max_depth=8, nee_mode=2, light_pick=1, bins=20, max_leaf=8))


def batch_scenes(seed: int = 0, n_scenes: int = 32, min_tris: float = 1e4, max_tris: float = 2e6,
                 resolutions=((256, 256), (512, 512), (1280, 720), (1920, 1080))):
    """The mixed batch: each scene = a displaced icosphere at the largest level
    under the drawn triangle count, a displaced ground grid topping the count
    up, and one emissive patch; resolution and bounce count (1..8) drawn per scene."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_scenes):
        target = int(math.exp(rng.uniform(math.log(min_tris), math.log(max_tris))))
        level = max(0, int(math.floor(math.log(max(target / 20.0, 1.0), 4))))
        while 20 * 4 ** level > target and level > 0:
            level -= 1
        rest = max(target - 20 * 4 ** level, 2)
        g = max(2, int(math.sqrt(rest / 2.0)) + 1)
        radius = sphere_radius_for(level)
        sphere = displaced_icosphere(level, 0.1, seed * 1000 + s, radius=radius)
        ground_size = max(12.0, 0.03 * (g - 1), 6.0 * radius)
        ground = fbm_grid(g, ground_size, 0.05 * ground_size, seed * 1000 + s, octaves=3)
        patch = disc_mesh(16, max(1.0, radius))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        depth = int(rng.integers(1, 9))
        mats = [Material((*rng.uniform(0.2, 0.9, 3), 1), (0, 0, 0, 1), rng.uniform(0.05, 1.0), 0.5,
                         float(rng.random() < 0.3)),
                Material((0.6, 0.6, 0.6, 1), (0, 0, 0, 1), 0.9, 0.5, 0.0),
                Material((0.8, 0.8, 0.8, 1), (10.0, 10.0, 10.0, 1), 1.0, 0.5, 0.0)]
        inst = [Instance(0, 0, trs((0, 0.2 * radius, 0), random_rotation(rng))),
                Instance(1, 1, trs((0, -1.2 * radius, 0))),
                Instance(2, 2, trs((0, 3.0 * radius, 0)))]
        view = bevy_view((0.0, 0.8 * radius, 4.5 * radius), (0.0, 0.0, 0.0), aspect=w / h)
        desc = SceneDesc(f"batch{s}", [sphere, ground, patch], mats, inst, view, w, h,
                         dict(max_depth=depth, nee_mode=2, light_pick=1, bins=20, max_leaf=8, seed=s))
        out.append(desc)
    return out


def terrain_scene(n: int = 4096, rock_level: int = 5, n_rocks: int = 4096, n_light_instances: int = 50,
                  tris_per_light: int = 200, seed: int = 0, width: int = 3840, height: int = 2160) -> SceneDesc:
    """fBm terrain of n^2 vertices (2(n-1)^2 triangles) plus n_rocks instances of
    a displaced icosphere rock (20*4^rock_level triangles) and emissive discs
    (n_light_instances x tris_per_light triangles) of radiance log-uniform in [0.5, 50]."""
    rng = np.random.default_rng(seed)
    size = 400.0
    terrain = fbm_grid(n, size, 12.0, seed)
    rock = displaced_icosphere(rock_level, 0.3, seed + 7, freq=2.0)
    light = disc_mesh(tris_per_light, 2.0)
    meshes = [terrain, rock, light]
    materials = [Material((0.45, 0.4, 0.35, 1), (0, 0, 0, 1), rng.uniform(0.02, 1.0), 0.5, 0.0)]
    instances = [Instance(0, 0)]
    for i in range(n_rocks):
        materials.append(Material((*rng.uniform(0.2, 0.7, 3), 1), (0, 0, 0, 1), rng.uniform(0.02, 1.0), 0.5, 0.0))
        pos = (rng.uniform(-size / 2.2, size / 2.2), rng.uniform(-6, 10), rng.uniform(-size / 2.2, size / 2.2))
        instances.append(Instance(1, len(materials) - 1, trs(pos, random_rotation(rng), rng.uniform(0.5, 3.0))))
    for i in range(n_light_instances):
        le = math.exp(rng.uniform(math.log(0.5), math.log(50.0)))
        materials.append(Material((0.8, 0.8, 0.8, 1), (le, le, le, 1), 1.0, 0.5, 0.0))
        pos = (rng.uniform(-size / 2.5, size / 2.5), 40.0, rng.uniform(-size / 2.5, size / 2.5))
        instances.append(Instance(2, len(materials) - 1, trs(pos)))
    view = bevy_view((0.0, 60.0, 220.0), (0.0, 0.0, 0.0), aspect=width / height)
    return SceneDesc("terrain", meshes, materials, instances, view, width, height,
                     dict(max_depth=16, nee_mode=2, light_pick=1, bins=32, max_leaf=4))
