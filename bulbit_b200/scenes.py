"""Procedural scenes and ray sets for the renderer's workloads.

Every scene is plain data (numpy arrays plus the ctypes records of
include/bbg.h) so the same bytes can be handed to the GPU library and, in the
tests, to the reference renderer. Random numbers come from PCG32 (the
generator of the reference's RNG, include/bulbit/random.h:27-46) run as one
independent stream per element (stream = element index), vectorised in numpy,
so every generator is deterministic for a seed and independent of how it is
batched.

Workloads (sizes as the benchmark configurations state them):
  readme_sphere()      the reference README scene: one red diffuse sphere, a
                       spot light and a uniform infinite light, 320x180
  triangle_soup()      ray-throughput scene: N triangles, centroids U[-1,1]^3,
                       vertices centroid + N(0, 0.01^2) per axis
  soup_rays()          rays from the sphere of radius 3 toward U[-1,1]^3
  cornell_icosphere()  closed 2x2x2 Cornell box (12 triangles) with a
                       0.5x0.5 one-sided ceiling light and a displaced gold
                       icosphere (20*4^L triangles)
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

F32 = np.float32
EPS32 = np.finfo(np.float32).eps
_MULT = np.uint64(0x5851F42D4C957F2D)


# ------------------------------------------------------------------ PCG32

class PCG32Streams:
    """n independent PCG32 generators, RNG(initstate, initseq=stream id)."""

    def __init__(self, initstate, streams):
        with np.errstate(over="ignore"):
            streams = np.asarray(streams, dtype=np.uint64)
            self.inc = (streams << np.uint64(1)) | np.uint64(1)
            self.state = np.zeros_like(streams)
            self._step()
            self.state = self.state + np.uint64(initstate)
            self._step()

    def _step(self):
        old = self.state
        with np.errstate(over="ignore"):
            self.state = old * _MULT + self.inc
        return old

    def next_uint(self):
        old = self._step()
        xorshifted = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
        rot = (old >> np.uint64(59)).astype(np.uint32)
        return (xorshifted >> rot) | (xorshifted << ((np.uint32(0) - rot) & np.uint32(31)))

    def next_float(self):
        u = self.next_uint().astype(np.float32) * F32(2.0 ** -32)
        return np.minimum(F32(1.0) - EPS32, u)


def _normalize_rows(v):
    """Normalize(v) of include/bulbit/math.h:56 in float32, row-wise."""
    v = v.astype(np.float32)
    l2 = v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]
    l2 = l2 + v[:, 2] * v[:, 2]
    inv = F32(1.0) / np.sqrt(l2)
    return v * inv[:, None]


def _f32_normalize(v):
    return _normalize_rows(np.asarray(v, np.float32)[None, :])[0]


def _f32_dist(a, b):
    d = np.asarray(b, np.float32) - np.asarray(a, np.float32)
    l2 = d[0] * d[0] + d[1] * d[1]
    l2 = l2 + d[2] * d[2]
    return F32(np.sqrt(F32(l2)))


# ------------------------------------------------------------------ scene data

@dataclass
class SceneData:
    positions: np.ndarray = None
    normals: np.ndarray = None
    tangents: np.ndarray = None
    uvs: np.ndarray = None
    tri_indices: np.ndarray = None
    spheres: list = field(default_factory=list)
    prim_kind: np.ndarray = None
    prim_index: np.ndarray = None
    prim_material: np.ndarray = None
    materials: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    camera: abi.CameraSpec = None
    spp: int = 1
    seed: int = 0
    max_bounces: int = 8
    rr_min_bounces: int = 1
    name: str = ""

    @property
    def n_prims(self):
        return 0 if self.prim_kind is None else int(self.prim_kind.shape[0])

    @property
    def n_triangles(self):
        return 0 if self.tri_indices is None else int(self.tri_indices.shape[0])

    def geometry(self):
        """A ctypes bbg_geometry viewing this scene's arrays (keep self alive)."""
        g = abi.Geometry()
        keep = []

        def ptr(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype)
            keep.append(a)
            return a.ctypes.data

        nv = 0 if self.positions is None else self.positions.shape[0]
        g.n_vertices = nv
        g.positions = ptr(self.positions, np.float32)
        g.normals = ptr(self.normals, np.float32)
        g.tangents = ptr(self.tangents, np.float32)
        g.uvs = ptr(self.uvs, np.float32)
        g.n_triangles = self.n_triangles
        g.tri_indices = ptr(self.tri_indices, np.int32)
        sph = (abi.Sphere * max(1, len(self.spheres)))(*self.spheres)
        keep.append(sph)
        g.n_spheres = len(self.spheres)
        g.spheres = C_addr(sph) if self.spheres else None
        g.n_prims = self.n_prims
        g.prim_kind = ptr(self.prim_kind, np.int32)
        g.prim_index = ptr(self.prim_index, np.int32)
        g._keep = keep
        return g

    def material_array(self):
        return (abi.Material * max(1, len(self.materials)))(*self.materials)

    def light_array(self):
        return (abi.Light * max(1, len(self.lights)))(*self.lights)


def C_addr(obj):
    import ctypes
    return ctypes.addressof(obj)


def diffuse(rgb):
    m = abi.Material()
    m.type = abi.BBG_MAT_DIFFUSE
    m.reflectance[:] = list(rgb)
    return m


def conductor(eta, k, roughness, reflectance=(1.0, 1.0, 1.0), energy_compensation=False):
    m = abi.Material()
    m.type = abi.BBG_MAT_CONDUCTOR
    m.eta[:] = list(eta)
    m.k[:] = list(k)
    m.roughness[:] = [roughness, roughness]
    m.reflectance[:] = list(reflectance)
    m.energy_compensation = 1 if energy_compensation else 0
    return m


def dielectric(ior, roughness=0.0, reflectance=(1.0, 1.0, 1.0), energy_compensation=False):
    m = abi.Material()
    m.type = abi.BBG_MAT_DIELECTRIC
    m.eta[:] = [ior, ior, ior]
    m.roughness[:] = [roughness, roughness]
    m.reflectance[:] = list(reflectance)
    m.energy_compensation = 1 if energy_compensation else 0
    return m


def metallic_roughness(basecolor, metallic, roughness):
    m = abi.Material()
    m.type = abi.BBG_MAT_METALLIC_ROUGHNESS
    m.reflectance[:] = list(basecolor)
    m.metallic = metallic
    m.roughness[:] = [roughness, roughness]
    return m


GOLD_ETA = (0.161, 0.492, 1.426)
GOLD_K = (4.08769, 2.32625, 1.846)


def camera_spec(position, target, up, vfov, aperture, focus, width, height, filter_extent=1.0,
                filter_type=abi.BBG_FILTER_BOX, filter_sigma=0.5):
    c = abi.CameraSpec()
    c.position[:] = list(position)
    c.target[:] = list(target)
    c.up[:] = list(up)
    c.vfov_deg = vfov
    c.aperture_radius = aperture
    c.focus_distance = float(focus)
    c.width = width
    c.height = height
    c.filter_extent = filter_extent
    c.filter_type = filter_type
    c.filter_sigma = filter_sigma
    return c


# ------------------------------------------------------------------ README scene

def readme_sphere(width=320, height=180, spp=16, max_bounces=8):
    """The reference README example (README.md "Bulbit as a standalone
    library"): sphere r=1 at (0,1,0), DiffuseMaterial (0.85,0.2,0.2), SpotLight
    at (2.5,4,2) aimed at the sphere (intensity 80, cone 35/20 deg),
    UniformInfiniteLight 0.1, camera at (3,2,5), fov 35, aperture 0.01,
    focus on the sphere, BoxFilter, IndependentSampler."""
    s = SceneData(name="readme_sphere")
    sph = abi.Sphere()
    sph.p[:] = [0.0, 1.0, 0.0]
    sph.q[:] = [0.0, 0.0, 0.0, 1.0]
    sph.s[:] = [1.0, 1.0, 1.0]
    sph.radius = 1.0
    s.spheres = [sph]
    s.prim_kind = np.array([abi.BBG_PRIM_SPHERE], np.int32)
    s.prim_index = np.array([0], np.int32)
    s.prim_material = np.array([0], np.int32)
    s.materials = [diffuse((0.85, 0.2, 0.2))]

    light_pos = np.array([2.5, 4.0, 2.0], np.float32)
    sphere_pos = np.array([0.0, 1.0, 0.0], np.float32)
    spot = abi.Light()
    spot.type = abi.BBG_LIGHT_SPOT
    spot.position[:] = light_pos.tolist()
    spot.direction[:] = _f32_normalize(light_pos - sphere_pos).tolist()
    spot.intensity[:] = [80.0, 80.0, 80.0]
    spot.angle_max = 35.0
    spot.angle_falloff_start = 20.0
    inf = abi.Light()
    inf.type = abi.BBG_LIGHT_UNIFORM_INFINITE
    inf.intensity[:] = [0.1, 0.1, 0.1]
    inf.scale = 1.0
    s.lights = [spot, inf]

    cam_pos = np.array([3.0, 2.0, 5.0], np.float32)
    s.camera = camera_spec(cam_pos, sphere_pos, (0.0, 1.0, 0.0), 35.0, 0.01,
                           _f32_dist(cam_pos, sphere_pos), width, height)
    s.spp, s.seed, s.max_bounces = spp, 0, max_bounces
    return s


# ------------------------------------------------------------------ triangle soup

def _gaussian_pairs(rng, sigma):
    """SampleGaussian (include/bulbit/sampling.h:14-21): Box-Muller on two
    uniforms, in float32."""
    u0 = rng.next_float()
    u1 = rng.next_float()
    r = F32(sigma) * np.sqrt(F32(-2.0) * np.log(np.maximum(u0, F32(1e-8))))
    theta = F32(2.0 * math.pi) * u1
    return r * np.cos(theta), r * np.sin(theta)


def triangle_soup(n_tris, seed=1, sigma=0.01):
    """n_tris triangles: centroid U[-1,1]^3, each vertex centroid + N(0,
    sigma^2) per axis; a triangle soup mesh (3 vertices per triangle) with face
    normals, first-edge tangents and zero uvs."""
    rng = PCG32Streams(seed, np.arange(n_tris, dtype=np.uint64))
    c = np.stack([F32(-1.0) + F32(2.0) * rng.next_float() for _ in range(3)], axis=1)
    g = []
    for _ in range(5):
        a, b = _gaussian_pairs(rng, sigma)
        g.extend([a, b])
    g = np.stack(g[:9], axis=1).reshape(n_tris, 3, 3)
    verts = (c[:, None, :] + g).astype(np.float32)
    pos = verts.reshape(-1, 3)
    e1 = verts[:, 1] - verts[:, 0]
    e2 = verts[:, 2] - verts[:, 0]
    n = _normalize_rows(np.cross(e1, e2))
    t = _normalize_rows(e1)
    s = SceneData(name=f"soup{n_tris}")
    s.positions = pos
    s.normals = np.repeat(n, 3, axis=0)
    s.tangents = np.repeat(t, 3, axis=0)
    s.uvs = np.zeros((pos.shape[0], 2), np.float32)
    s.tri_indices = np.arange(3 * n_tris, dtype=np.int32).reshape(n_tris, 3)
    s.prim_kind = np.zeros(n_tris, np.int32)
    s.prim_index = np.arange(n_tris, dtype=np.int32)
    s.prim_material = np.full(n_tris, -1, np.int32)
    return s


def soup_rays(n_rays, seed=2, radius=3.0):
    """n_rays rays: origin uniform on the sphere of the given radius
    (SampleUniformSphere, include/bulbit/sampling.h:59-70), direction toward a
    uniform point of [-1,1]^3, normalised. Returns (closest, any): closest
    queries use [1e-4, inf]; any-hit queries [1e-4, 0.5*distance]."""
    rng = PCG32Streams(seed, np.arange(n_rays, dtype=np.uint64))
    u0 = rng.next_float()
    u1 = rng.next_float()
    z = F32(1.0) - F32(2.0) * u0
    r = np.sqrt(np.maximum(F32(0.0), F32(1.0) - z * z))
    phi = F32(2.0 * math.pi) * u1
    o = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32) * F32(radius)
    tgt = np.stack([F32(-1.0) + F32(2.0) * rng.next_float() for _ in range(3)], axis=1)
    v = (tgt - o).astype(np.float32)
    l2 = v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]
    l2 = l2 + v[:, 2] * v[:, 2]
    dist = np.sqrt(l2)
    d = v * (F32(1.0) / dist)[:, None]
    closest = np.zeros((n_rays, 8), np.float32)
    closest[:, 0:3] = o
    closest[:, 3:6] = d
    closest[:, 6] = F32(1e-4)
    closest[:, 7] = np.inf
    anyq = closest.copy()
    anyq[:, 7] = F32(0.5) * dist
    return closest, anyq


# ------------------------------------------------------------------ Cornell box

def icosphere(levels):
    """Unit icosphere: icosahedron subdivided `levels` times (each triangle
    into four, midpoints pushed to the sphere). Returns (vertices float64,
    faces int32)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1)[:, None]
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(levels):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (1 << 32) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq >> 32
        b = uniq & ((1 << 32) - 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1)[:, None]
        base = v.shape[0]
        v = np.concatenate([v, mid], axis=0)
        nf = f.shape[0]
        m01 = base + inv[0:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:3 * nf]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)], axis=0)
    return v, f.astype(np.int32)


def geodesic_sphere(freq):
    """Unit geodesic sphere of any frequency: every icosahedron face divided
    into freq^2 triangles on a barycentric grid, points pushed to the sphere
    (20 freq^2 triangles, 10 freq^2 + 2 vertices). Returns (vertices float64,
    faces int32)."""
    v0, f0 = icosphere(0)
    n = int(freq)
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = ii + jj <= n
    ii, jj = ii[keep], jj[keep]
    local = -np.ones((n + 1, n + 1), np.int64)
    local[ii, jj] = np.arange(ii.size)
    # Triangles of one face in grid indices (both orientations of cells).
    ti, tj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = ti + tj < n
    dn = ti + tj < n - 1
    tri_up = np.stack([local[ti[up], tj[up]], local[ti[up] + 1, tj[up]], local[ti[up], tj[up] + 1]], 1)
    tri_dn = np.stack([local[ti[dn] + 1, tj[dn]], local[ti[dn] + 1, tj[dn] + 1], local[ti[dn], tj[dn] + 1]], 1)
    tris = np.concatenate([tri_up, tri_dn], 0)
    pts, faces = [], []
    for k, (a, b, c) in enumerate(f0):
        p = v0[a] + (v0[b] - v0[a]) * (ii[:, None] / n) + (v0[c] - v0[a]) * (jj[:, None] / n)
        pts.append(p / np.linalg.norm(p, axis=1)[:, None])
        faces.append(tris + k * ii.size)
    pts = np.concatenate(pts, 0)
    faces = np.concatenate(faces, 0)
    # Merge the copies of points on shared edges and corners.
    key = np.round(pts * 1e9).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    return pts[first], inv.reshape(-1)[faces].astype(np.int32)


def _vertex_normals(pos, faces):
    p = pos.astype(np.float64)
    fn = np.cross(p[faces[:, 1]] - p[faces[:, 0]], p[faces[:, 2]] - p[faces[:, 0]])
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, faces[:, k], fn)
    n /= np.linalg.norm(n, axis=1)[:, None]
    return n


def _tangents(n):
    a = np.where(np.abs(n[:, 1:2]) < 0.999, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(a, n)
    return t / np.linalg.norm(t, axis=1)[:, None]


CORNELL_RED = (0.63, 0.065, 0.05)
CORNELL_GREEN = (0.14, 0.45, 0.091)
CORNELL_WHITE = (0.725, 0.71, 0.68)


def cornell_icosphere(levels=8, width=1024, height=1024, spp=64, max_bounces=16, seed=3, freq=None,
                      displacement=0.02, sphere_material=None, light_emission=(17.0, 12.0, 4.0)):
    """Closed Cornell box [-1,1]^3 (12 triangles: left wall red, right wall
    green, floor/ceiling/back/front white), a 0.5x0.5 one-sided diffuse area
    light just under the ceiling facing down (2 triangles, one DiffuseAreaLight
    each), and an icosphere of radius 0.5 resting on the floor, `levels`
    subdivisions, each vertex displaced radially by N(0, displacement^2),
    gold conductor of roughness 0.2 unless sphere_material is given. The
    camera sits inside the box near the front wall, looking at the back wall."""
    s = SceneData(name=f"cornell_ico{levels}" if freq is None else f"cornell_geo{freq}")
    mats = [diffuse(CORNELL_RED), diffuse(CORNELL_GREEN), diffuse(CORNELL_WHITE),
            sphere_material or conductor(GOLD_ETA, GOLD_K, 0.2)]
    RED, GREEN, WHITE, SPHERE = 0, 1, 2, 3

    # Box: 6 quads, each 2 triangles, wound so the normal faces the interior.
    P = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)
    quads = [([0, 4, 7, 3], RED),    # left  x=-1, normal +x
             ([1, 2, 6, 5], GREEN),  # right x=+1, normal -x
             ([0, 1, 5, 4], WHITE),  # floor y=-1, normal +y
             ([3, 7, 6, 2], WHITE),  # ceiling y=+1, normal -y
             ([0, 3, 2, 1], WHITE),  # back z=-1, normal +z
             ([4, 5, 6, 7], WHITE)]  # front z=+1, normal -z
    pos, nrm, tri, tmat = [], [], [], []
    for q, m in quads:
        a, b, c, d = (P[i] for i in q)
        n = np.cross(b - a, c - a)
        if np.dot(n, -a) < 0:  # wind so the geometric normal faces the interior
            a, b, c, d = a, d, c, b
            n = -n
        n /= np.linalg.norm(n)
        base = len(pos)
        pos.extend([a, b, c, d])
        nrm.extend([n] * 4)
        tri.extend([[base, base + 1, base + 2], [base, base + 2, base + 3]])
        tmat.extend([m, m])
    # Light quad at y = 0.999, facing down, 0.5 x 0.5.
    h = 0.25
    ly = 0.999
    la, lb, lc, ld = (np.array(p, np.float64) for p in
                      ([-h, ly, -h], [h, ly, -h], [h, ly, h], [-h, ly, h]))
    n = np.cross(lb - la, lc - la)
    n /= np.linalg.norm(n)  # (0,-1,0)
    base = len(pos)
    pos.extend([la, lb, lc, ld])
    nrm.extend([n] * 4)
    light_tris = [len(tri), len(tri) + 1]
    tri.extend([[base, base + 1, base + 2], [base, base + 2, base + 3]])
    tmat.extend([WHITE, WHITE])

    box_pos = np.array(pos)
    box_nrm = np.array(nrm)
    box_tri = np.array(tri, np.int64)

    # Icosphere.
    v, f = icosphere(levels) if freq is None else geodesic_sphere(freq)
    rng = PCG32Streams(seed, np.arange(v.shape[0], dtype=np.uint64))
    g, _ = _gaussian_pairs(rng, displacement)
    radius = 0.5 + g.astype(np.float64)
    center = np.array([0.0, -0.5, 0.0])
    sp = center + v * radius[:, None]
    sn = _vertex_normals(sp, f)

    all_pos = np.concatenate([box_pos, sp], 0)
    all_nrm = np.concatenate([box_nrm, sn], 0)
    all_tan = _tangents(all_nrm)
    all_tri = np.concatenate([box_tri, f.astype(np.int64) + box_pos.shape[0]], 0)
    n_tris = all_tri.shape[0]

    s.positions = all_pos.astype(np.float32)
    s.normals = _normalize_rows(all_nrm.astype(np.float32))
    s.tangents = _normalize_rows(all_tan.astype(np.float32))
    s.uvs = np.zeros((all_pos.shape[0], 2), np.float32)
    s.tri_indices = all_tri.astype(np.int32)
    s.prim_kind = np.zeros(n_tris, np.int32)
    s.prim_index = np.arange(n_tris, dtype=np.int32)
    s.prim_material = np.concatenate([np.array(tmat, np.int32),
                                      np.full(f.shape[0], SPHERE, np.int32)])
    s.materials = mats
    for t in light_tris:
        l = abi.Light()
        l.type = abi.BBG_LIGHT_DIFFUSE_AREA
        l.prim = t
        l.two_sided = 0
        l.intensity[:] = list(light_emission)
        s.lights.append(l)

    s.camera = camera_spec((0.0, 0.0, 0.98), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 70.0, 0.0, 1.0,
                           width, height)
    s.spp, s.seed, s.max_bounces = spp, 0, max_bounces
    return s


BATCH_RESOLUTIONS = (256, 512, 768, 1024)


def cornell_batch_variant(seed, spp=32, max_bounces=12, resolution=None):
    """One of the uneven Cornell-box variants rendered as a batch: the sphere
    is a displaced geodesic sphere whose triangle count is drawn log-uniform
    in [10^4, 2x10^6] (frequency round(sqrt(count / 20))), its material drawn
    uniformly from {Lambertian albedo U(0.2, 0.9) per channel, smooth
    dielectric IOR 1.5, gold conductor roughness U(0.05, 0.5)}, and the
    resolution from 256^2 .. 1024^2; all draws from numpy's generator seeded
    with `seed`, the displacement from PCG32 seeded with it."""
    rng = np.random.default_rng(seed)
    count = math.exp(rng.uniform(math.log(1e4), math.log(2e6)))
    freq = max(1, int(round(math.sqrt(count / 20))))
    kind = int(rng.integers(3))
    if kind == 0:
        mat = diffuse(tuple(float(x) for x in rng.uniform(0.2, 0.9, 3)))
    elif kind == 1:
        mat = dielectric(1.5)
    else:
        mat = conductor(GOLD_ETA, GOLD_K, float(rng.uniform(0.05, 0.5)))
    res = int(rng.choice(BATCH_RESOLUTIONS)) if resolution is None else resolution
    s = cornell_icosphere(width=res, height=res, spp=spp, max_bounces=max_bounces, seed=seed, freq=freq,
                          sphere_material=mat)
    s.name = f"variant{seed}:geo{freq}:{['lambertian', 'dielectric', 'conductor'][kind]}:{res}"
    return s
