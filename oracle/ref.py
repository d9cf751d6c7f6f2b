"""ctypes wrapper of the oracle harness (oracle/_ref/libbulbit_ref.so).

TEST INFRASTRUCTURE ONLY: the reference renderer compiled from its own
sources, used by tests/ and by the CPU-baseline leg of bench.py to check and
time the GPU library. Nothing in the product imports this module.
"""
import ctypes as C
import os

import numpy as np

from bulbit_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libbulbit_ref.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        sig = {
            "bbref_init": (I32, [I32]),
            "bbref_scene_create": (P, [P, P, P, I32, P, I32, P]),
            "bbref_scene_destroy": (None, [P]),
            "bbref_integrator_create": (I32, [P, I32, I32, I32, I32, I32, P]),
            "bbref_bvh_node_count": (I32, [P]),
            "bbref_bvh_export": (I32, [P, P, P]),
            "bbref_mesh_export": (I32, [P, P, P, P, P]),
            "bbref_intersect": (C.c_double, [P, P, I64, P]),
            "bbref_intersect_any": (C.c_double, [P, P, I64, P]),
            "bbref_intersect_all": (I32, [P, P, I32, P, P]),
            "bbref_camera": (I32, [P, P]),
            "bbref_trace_paths": (C.c_double, [P, P, I32, I32, P, I64, P]),
            "bbref_render": (C.c_double, [P, P, P, P]),
            "bbref_light_pmf": (I32, [P, P]),
            "bbref_sampler_draws": (I32, [I32, I32, I32, I32, I32, P]),
            "bbref_ggx_energy_tables": (I32, [P, P]),
            "bbref_dielectric_energy_tables": (I32, [P, P, P, P]),
            "bbref_count_traversal": (I32, [P, P, C.c_int64, I32, P, P]),
            "bbref_bsdf_probe": (I32, [P, I32, I32, P, P, P, P]),
            "bbref_set_sampler": (None, [I32, I32, I32]),
            "bbref_pcg32": (I32, [C.c_uint64, C.c_uint64, I32, P]),
            "bbref_hash_pixel_sample": (C.c_uint64, [I32, I32, I32, I32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def init(threads=0):
    return lib().bbref_init(threads)


def _p(a):
    return a.ctypes.data


class RefScene:
    """A reference Scene + BVH (+ PathIntegrator on demand) built from SceneData."""

    def __init__(self, scene):
        self.scene = scene
        g = scene.geometry()
        mats = scene.material_array()
        lights = scene.light_array()
        pm = np.ascontiguousarray(scene.prim_material, np.int32)
        secs = C.c_double()
        self.h = lib().bbref_scene_create(C.byref(g), _p(pm), C.addressof(mats), len(scene.materials),
                                          C.addressof(lights), len(scene.lights), C.byref(secs))
        self.build_seconds = secs.value
        self.integrator_seconds = None

    def close(self):
        if self.h:
            lib().bbref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def make_integrator(self, spp=None, seed=None, max_bounces=None, rr_min_bounces=None, regularize=0):
        s = self.scene
        secs = C.c_double()
        lib().bbref_integrator_create(self.h, spp or s.spp, s.seed if seed is None else seed,
                                      s.max_bounces if max_bounces is None else max_bounces,
                                      s.rr_min_bounces if rr_min_bounces is None else rr_min_bounces,
                                      regularize, C.byref(secs))
        self.integrator_seconds = secs.value

    def bvh(self):
        n = lib().bbref_bvh_node_count(self.h)
        nodes = np.zeros(n, dtype=np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("offset", "<i4"),
                                            ("count", "<u2"), ("axis", "u1"), ("pad", "u1")]))
        slots = np.zeros(self.scene.n_prims, np.int32)
        lib().bbref_bvh_export(self.h, _p(nodes), _p(slots))
        return nodes, slots

    def mesh_arrays(self):
        nv = self.scene.positions.shape[0]
        pos = np.zeros((nv, 3), np.float32)
        nrm = np.zeros((nv, 3), np.float32)
        tan = np.zeros((nv, 3), np.float32)
        uv = np.zeros((nv, 2), np.float32)
        lib().bbref_mesh_export(self.h, _p(pos), _p(nrm), _p(tan), _p(uv))
        return pos, nrm, tan, uv

    def intersect(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 4), np.float32)
        secs = lib().bbref_intersect(self.h, _p(rays), rays.shape[0], _p(hits))
        return hits[:, 0].view(np.int32).copy(), hits[:, 1].copy(), secs

    def intersect_any(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint8)
        secs = lib().bbref_intersect_any(self.h, _p(rays), rays.shape[0], _p(occ))
        return occ, secs

    def count_traversal(self, rays, any_hit=False):
        """Nodes popped and primitive tests of BVH::RayCast over the rays (totals)."""
        rays = np.ascontiguousarray(rays, np.float32)
        nodes, prims = C.c_int64(), C.c_int64()
        lib().bbref_count_traversal(self.h, _p(rays), rays.shape[0], 1 if any_hit else 0, C.byref(nodes),
                                    C.byref(prims))
        return nodes.value, prims.value

    def intersect_all(self, ray, max_out=64):
        ray = np.ascontiguousarray(ray, np.float32)
        prims = np.zeros(max_out, np.int32)
        ts = np.zeros(max_out, np.float32)
        n = lib().bbref_intersect_all(self.h, _p(ray), max_out, _p(prims), _p(ts))
        n = min(n, max_out)
        order = np.argsort(ts[:n], kind="stable")
        return prims[:n][order], ts[:n][order]

    def trace_paths(self, path_ids=None, spp=None):
        s = self.scene
        spp = spp or s.spp
        cam = s.camera
        if path_ids is None:
            n = cam.width * cam.height * spp
            ids_ptr = None
        else:
            path_ids = np.ascontiguousarray(path_ids, np.int64)
            n = path_ids.shape[0]
            ids_ptr = _p(path_ids)
        L = np.zeros((n, 3), np.float32)
        secs = lib().bbref_trace_paths(self.h, C.byref(cam), spp, s.seed, ids_ptr, n, _p(L))
        return L, secs

    def render(self):
        cam = self.scene.camera
        img = np.zeros((cam.height, cam.width, 3), np.float32)
        var = np.zeros((cam.height, cam.width), np.float32)
        secs = lib().bbref_render(self.h, C.byref(cam), _p(img), _p(var))
        return img, var, secs

    def light_pmf(self):
        out = np.zeros(max(1, len(self.scene.lights)), np.float32)
        lib().bbref_light_pmf(self.h, _p(out))
        return out[:len(self.scene.lights)]


def camera(spec):
    out = abi.Camera()
    lib().bbref_camera(C.byref(spec), C.byref(out))
    return out


def sampler_draws(px, py, seed, sample, n):
    out = np.zeros(n, np.float32)
    lib().bbref_sampler_draws(px, py, seed, sample, n, _p(out))
    return out


def set_sampler(kind=0, x_samples=1, jitter=1):
    """Sampler for later integrators and path traces: 0 independent, 1 stratified."""
    lib().bbref_set_sampler(kind, x_samples, jitter)


def ggx_energy_tables():
    """The reference's GGX energy tables: (E 32x32 indexed [alpha][cos], E_avg 32)."""
    e = np.zeros(32 * 32, np.float32)
    a = np.zeros(32, np.float32)
    lib().bbref_ggx_energy_tables(_p(e), _p(a))
    return e.reshape(32, 32), a


def dielectric_energy_tables():
    """The reference's rough-dielectric energy tables: (E, E_inv) 32x32x32
    indexed [alpha][cos][f0], (E_avg, E_inv_avg) 32x32 indexed [alpha][f0]."""
    e = np.zeros(32 ** 3, np.float32)
    ei = np.zeros(32 ** 3, np.float32)
    a = np.zeros(32 * 32, np.float32)
    ai = np.zeros(32 * 32, np.float32)
    lib().bbref_dielectric_energy_tables(_p(e), _p(ei), _p(a), _p(ai))
    return e.reshape(32, 32, 32), ei.reshape(32, 32, 32), a.reshape(32, 32), ai.reshape(32, 32)


def bsdf_probe(material, wo, wi, u, front_face=True):
    """The reference's Material::GetBSDF then f / PDF / Sample_f (bbg_bsdf_probe's layout)."""
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    out = np.zeros((wo.shape[0], 12), np.float32)
    rc = lib().bbref_bsdf_probe(C.byref(material), 1 if front_face else 0, wo.shape[0], _p(wo), _p(wi), _p(u),
                                _p(out))
    assert rc == 0
    return out


def pcg32(initstate, initseq, n):
    out = np.zeros(n, np.uint32)
    lib().bbref_pcg32(initstate, initseq, n, _p(out))
    return out


def hash_pixel_sample(px, py, seed, sample):
    return lib().bbref_hash_pixel_sample(px, py, seed, sample)
