"""Python binding of libbulbit_b200.so (include/bbg.h) for tests and benchmarks.

The GPU library is required: if the shared library is missing or a call fails,
an exception is raised — there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbulbit_b200.so")

_lib = None


class BbgError(RuntimeError):
    def __init__(self, status, where):
        msg = get_lib().bbg_last_error().decode(errors="replace")
        super().__init__(f"{where}: {abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def get_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"bulbit_b200 native library not built: {LIB_PATH} "
                               "(python -c 'import __graft_entry__ as g; g.build()')")
        L = C.CDLL(LIB_PATH)
        for name, res, args in abi.EXPORTS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, where):
    if status != abi.BBG_OK:
        raise BbgError(status, where)


def _p(a):
    return None if a is None else a.ctypes.data


def _dev_ptr(t):
    return C.c_void_p(t.data_ptr())


def bvh_build(aabbs):
    """bbg_bvh_build over (n, 6) float32 AABBs -> (nodes, slot_prims)."""
    aabbs = np.ascontiguousarray(aabbs, np.float32)
    n = aabbs.shape[0]
    nodes = np.zeros(max(1, 2 * n - 1), dtype=NODE_DTYPE)
    slots = np.zeros(n, np.int32)
    nn = C.c_int32()
    check(get_lib().bbg_bvh_build(_p(aabbs), n, _p(nodes), _p(slots), C.byref(nn)), "bbg_bvh_build")
    return nodes[:nn.value].copy(), slots


def prim_aabbs(scene):
    g = scene.geometry()
    out = np.zeros((scene.n_prims, 6), np.float32)
    check(get_lib().bbg_prim_aabbs(C.byref(g), _p(out)), "bbg_prim_aabbs")
    return out


def split_references(scene, budget):
    """bbg_split_references: (reference boxes (m, 6), their primitives (m,))."""
    g = scene.geometry()
    cap = int(scene.n_prims * (1 + budget)) + 1
    boxes = np.zeros((cap, 6), np.float32)
    prims = np.zeros(cap, np.int32)
    n = C.c_int32()
    check(get_lib().bbg_split_references(C.byref(g), float(budget), cap, _p(boxes), _p(prims), C.byref(n)),
          "bbg_split_references")
    return boxes[:n.value].copy(), prims[:n.value].copy()


def camera(spec):
    out = abi.Camera()
    check(get_lib().bbg_camera_perspective(C.byref(spec), C.byref(out)), "bbg_camera_perspective")
    return out


NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("offset", "<i4"),
                       ("count", "<u2"), ("axis", "u1"), ("pad", "u1")])


class GpuAccel:
    """The GPU accel beside the reference BVH (bbg_accel_*)."""

    def __init__(self, scene, bvh=None, device_build=False, split=None, device_sah=False):
        """bvh: the reference's tree (nodes, slots); device_build: the linear BVH
        built on the device; device_sah: the reference's SAH tree built on the
        device (bbg_accel_create_device_sah); split: extra references per
        primitive for the split-reference SAH build (bbg_accel_create_split,
        or bbg_accel_create_device_split with device_sah)."""
        self.scene = scene
        self._g = scene.geometry()
        self.h = C.c_void_p()
        if device_sah and split is not None:
            check(get_lib().bbg_accel_create_device_split(C.byref(self._g), float(split), C.byref(self.h)),
                  "bbg_accel_create_device_split")
            return
        if device_sah:
            check(get_lib().bbg_accel_create_device_sah(C.byref(self._g), C.byref(self.h)),
                  "bbg_accel_create_device_sah")
            return
        if device_build:
            check(get_lib().bbg_accel_create_device_build(C.byref(self._g), C.byref(self.h)),
                  "bbg_accel_create_device_build")
            return
        if split is not None:
            check(get_lib().bbg_accel_create_split(C.byref(self._g), float(split), C.byref(self.h)),
                  "bbg_accel_create_split")
            return
        bvh_arg = None
        if bvh is not None:
            nodes, slots = bvh
            self._bvh_nodes = np.ascontiguousarray(nodes)
            self._bvh_slots = np.ascontiguousarray(slots, np.int32)
            b = abi.Bvh()
            b.n_nodes = self._bvh_nodes.shape[0]
            b.nodes = _p(self._bvh_nodes)
            b.n_slots = self._bvh_slots.shape[0]
            b.slot_prims = _p(self._bvh_slots)
            bvh_arg = C.byref(b)
            self._bvh_struct = b
        check(get_lib().bbg_accel_create(C.byref(self._g), bvh_arg, C.byref(self.h)), "bbg_accel_create")

    def close(self):
        if self.h:
            get_lib().bbg_accel_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bounds(self):
        out = np.zeros(6, np.float32)
        check(get_lib().bbg_accel_bounds(self.h, _p(out)), "bbg_accel_bounds")
        return out

    def export(self):
        nn, ns = C.c_int32(), C.c_int32()
        check(get_lib().bbg_accel_export(self.h, None, None, C.byref(nn), C.byref(ns)), "bbg_accel_export")
        nodes = np.zeros(nn.value, NODE_DTYPE)
        slots = np.zeros(ns.value, np.int32)
        check(get_lib().bbg_accel_export(self.h, _p(nodes), _p(slots), None, None), "bbg_accel_export")
        return nodes, slots

    def set_traversal(self, mode):
        """abi.BBG_TRAVERSAL_WIDE (default for host-built trees), abi.BBG_TRAVERSAL_ORDERED or
        abi.BBG_TRAVERSAL_REFERENCE."""
        check(get_lib().bbg_accel_set_traversal(self.h, mode), "bbg_accel_set_traversal")

    def export_wide8(self):
        """The 8-wide node layout as (n, 24) float32 (empty where not built)."""
        n = C.c_int32(0)
        check(get_lib().bbg_accel_export_wide8(self.h, None, C.byref(n)), "bbg_accel_export_wide8")
        out = np.zeros((n.value, 24), np.float32)
        if n.value:
            check(get_lib().bbg_accel_export_wide8(self.h, _p(out), C.byref(n)), "bbg_accel_export_wide8")
        return out

    def set_counting(self, on):
        check(get_lib().bbg_accel_set_counting(self.h, 1 if on else 0), "bbg_accel_set_counting")

    def last_counts(self):
        a, b = C.c_int64(), C.c_int64()
        check(get_lib().bbg_accel_last_counts(self.h, C.byref(a), C.byref(b)), "bbg_accel_last_counts")
        return a.value, b.value

    def intersect(self, rays):
        """Closest hits of (n, 8) float32 rays (host numpy) -> (prim, t, u, v)."""
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 4), np.float32)
        check(get_lib().bbg_intersect(self.h, _p(rays), rays.shape[0], _p(hits), abi.BBG_MEM_HOST, None),
              "bbg_intersect")
        return hits[:, 0].view(np.int32).copy(), hits[:, 1].copy(), hits[:, 2].copy(), hits[:, 3].copy()

    def intersect_any(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint8)
        check(get_lib().bbg_intersect_any(self.h, _p(rays), rays.shape[0], _p(occ), abi.BBG_MEM_HOST, None),
              "bbg_intersect_any")
        return occ

    def intersect_device(self, rays_t, hits_t, stream=None):
        """Device-resident query: rays_t (n, 8) float32 and hits_t (n, 4) torch CUDA tensors."""
        check(get_lib().bbg_intersect(self.h, _dev_ptr(rays_t), rays_t.shape[0], _dev_ptr(hits_t),
                                      abi.BBG_MEM_DEVICE, stream), "bbg_intersect")

    def intersect_any_device(self, rays_t, occ_t, stream=None):
        check(get_lib().bbg_intersect_any(self.h, _dev_ptr(rays_t), rays_t.shape[0], _dev_ptr(occ_t),
                                          abi.BBG_MEM_DEVICE, stream), "bbg_intersect_any")

    def intersect_host_ptr(self, rays_ptr, n, hits_ptr):
        check(get_lib().bbg_intersect(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr), abi.BBG_MEM_HOST,
                                      None), "bbg_intersect")

    def intersect_any_host_ptr(self, rays_ptr, n, occ_ptr):
        check(get_lib().bbg_intersect_any(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(occ_ptr), abi.BBG_MEM_HOST,
                                          None), "bbg_intersect_any")

    def submit_host_ptr(self, rays_ptr, n, hits_ptr):
        """bbg_intersect_submit over host buffers: returns once queued."""
        check(get_lib().bbg_intersect_submit(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr),
                                             abi.BBG_MEM_HOST), "bbg_intersect_submit")

    def submit_any_host_ptr(self, rays_ptr, n, occ_ptr):
        check(get_lib().bbg_intersect_any_submit(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(occ_ptr),
                                                 abi.BBG_MEM_HOST), "bbg_intersect_any_submit")

    def submit_device(self, rays_t, hits_t):
        check(get_lib().bbg_intersect_submit(self.h, _dev_ptr(rays_t), rays_t.shape[0], _dev_ptr(hits_t),
                                             abi.BBG_MEM_DEVICE), "bbg_intersect_submit")

    def submit_any_device(self, rays_t, occ_t):
        check(get_lib().bbg_intersect_any_submit(self.h, _dev_ptr(rays_t), rays_t.shape[0], _dev_ptr(occ_t),
                                                 abi.BBG_MEM_DEVICE), "bbg_intersect_any_submit")

    def synchronize(self):
        check(get_lib().bbg_accel_synchronize(self.h), "bbg_accel_synchronize")


def sampler_draws(px, py, seed, sample, n):
    out = np.zeros(n, np.float32)
    check(get_lib().bbg_sampler_draws(px, py, seed, sample, n, _p(out)), "bbg_sampler_draws")
    return out


class Film:
    """Per-pixel film state of a render (what Film::AddSample maintains)."""

    def __init__(self, width, height, spp, path_L=False):
        self.width, self.height, self.spp = width, height, spp
        self.rgb_sum = np.zeros((height, width, 3), np.float32)
        self.count = np.zeros((height, width), np.int32)
        self.moments = np.zeros((height, width, 2), np.float32)
        self.path_L = np.zeros((height * width * spp, 3), np.float32) if path_L else None
        self.stats = abi.RenderStats()

    def struct(self):
        f = abi.Film()
        f.rgb_sum = _p(self.rgb_sum)
        f.count = _p(self.count)
        f.moments = _p(self.moments)
        f.path_L = _p(self.path_L)
        return f

    def image(self):
        """Film::GetRenderedImage: sum / count (src/reconstruction/film.cpp:80-100)."""
        with np.errstate(invalid="ignore", divide="ignore"):
            return self.rgb_sum / self.count[..., None].astype(np.float32)


class GpuPathIntegrator:
    """PathIntegrator(accel, lights, sampler, max_bounces, rr_min_bounces,
    regularize_bsdf) on the GPU (bbg_integrator_*, bbg_render)."""

    def __init__(self, accel, scene, max_bounces=None, rr_min_bounces=None, regularize=0):
        self.accel = accel
        self.scene = scene
        self._mats = scene.material_array()
        self._lights = scene.light_array()
        self._pm = np.ascontiguousarray(scene.prim_material, np.int32)
        self.h = C.c_void_p()
        mb = scene.max_bounces if max_bounces is None else max_bounces
        rr = scene.rr_min_bounces if rr_min_bounces is None else rr_min_bounces
        check(get_lib().bbg_integrator_create(accel.h, _p(self._pm), C.addressof(self._mats), len(scene.materials),
                                              C.addressof(self._lights), len(scene.lights), mb, rr, regularize,
                                              C.byref(self.h)), "bbg_integrator_create")

    def close(self):
        if self.h:
            get_lib().bbg_integrator_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def light_pmf(self):
        out = np.zeros(max(1, len(self.scene.lights)), np.float32)
        check(get_lib().bbg_integrator_light_pmf(self.h, _p(out)), "bbg_integrator_light_pmf")
        return out[:len(self.scene.lights)]

    def render(self, spp=None, seed=None, camera_spec=None, wave_paths=0, use_graph=True, light_alias=False,
               path_L=False, guide=None, train=False, batch=0, lr=0.0, select=0.0, steps=0,
               sampler=abi.BBG_SAMPLER_INDEPENDENT, x_samples=1, jitter=True, shade_order=abi.BBG_SHADE_SORTED,
               pass_through_levels=0):
        s = self.scene
        spec = camera_spec or s.camera
        cam = camera(spec)
        spp = spp or s.spp
        p = abi.RenderParams()
        p.spp = spp
        p.seed = s.seed if seed is None else seed
        p.wave_paths = wave_paths
        p.use_graph = 1 if use_graph else 0
        p.light_alias = 1 if light_alias else 0
        p.guide = guide.h if guide is not None else None
        p.guide_train = 1 if train else 0
        p.guide_batch = batch
        p.guide_lr = lr
        p.guide_select = select
        p.guide_steps = steps
        p.sampler = sampler
        p.x_samples = x_samples
        p.jitter = 1 if jitter else 0
        p.shade_order = shade_order
        p.pass_through_levels = pass_through_levels
        film = Film(cam.width, cam.height, spp, path_L=path_L)
        fs = film.struct()
        check(get_lib().bbg_render(self.h, C.byref(cam), C.byref(p), C.byref(fs), abi.BBG_MEM_HOST,
                                   C.byref(film.stats)), "bbg_render")
        return film

    def autotune(self, spp=None, seed=None, camera_spec=None):
        """bbg_integrator_autotune for renders at spp -> abi.Tuning."""
        cam = camera(camera_spec or self.scene.camera)
        p = abi.RenderParams()
        p.spp = spp or self.scene.spp
        p.seed = self.scene.seed if seed is None else seed
        out = abi.Tuning()
        check(get_lib().bbg_integrator_autotune(self.h, C.byref(cam), C.byref(p), C.byref(out)),
              "bbg_integrator_autotune")
        return out

    def set_tuning(self, block=128, short_stack=16, wave_paths=0):
        t = abi.Tuning()
        t.block, t.short_stack, t.wave_paths = block, short_stack, wave_paths
        check(get_lib().bbg_integrator_set_tuning(self.h, C.byref(t)), "bbg_integrator_set_tuning")

    def render_device(self, cam, params, film_struct, stats):
        check(get_lib().bbg_render(self.h, C.byref(cam), C.byref(params), C.byref(film_struct),
                                   abi.BBG_MEM_DEVICE, C.byref(stats)), "bbg_render")


class GpuGuide:
    """The path-guiding MLP (bbg_guide_*)."""

    N_PARAMS = 16104

    def __init__(self, aabb, seed=1):
        self._aabb = np.ascontiguousarray(aabb, np.float32)
        self.h = C.c_void_p()
        check(get_lib().bbg_guide_create(_p(self._aabb), seed, C.byref(self.h)), "bbg_guide_create")

    def close(self):
        if self.h:
            get_lib().bbg_guide_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(self.N_PARAMS, np.float32)
        check(get_lib().bbg_guide_get_params(self.h, _p(out)), "bbg_guide_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(get_lib().bbg_guide_set_params(self.h, _p(p)), "bbg_guide_set_params")

    def forward(self, raw):
        raw = np.ascontiguousarray(raw, np.float32)
        out = np.zeros((raw.shape[0], 40), np.float32)
        check(get_lib().bbg_guide_forward(self.h, _p(raw), raw.shape[0], _p(out)), "bbg_guide_forward")
        return out

    def gradient(self, raw, dirs, weights):
        raw = np.ascontiguousarray(raw, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        weights = np.ascontiguousarray(weights, np.float32)
        g = np.zeros(self.N_PARAMS, np.float32)
        loss = C.c_float()
        check(get_lib().bbg_guide_gradient(self.h, _p(raw), _p(dirs), _p(weights), raw.shape[0], _p(g),
                                           C.byref(loss)), "bbg_guide_gradient")
        return g, loss.value

    def train_step(self, raw, dirs, weights, lr=1e-2):
        raw = np.ascontiguousarray(raw, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        weights = np.ascontiguousarray(weights, np.float32)
        loss = C.c_float()
        check(get_lib().bbg_guide_train_step(self.h, _p(raw), _p(dirs), _p(weights), raw.shape[0], C.c_float(lr),
                                             C.byref(loss)), "bbg_guide_train_step")
        return loss.value


class GpuBatch:
    """Several scenes rendered together (bbg_batch_*)."""

    def __init__(self):
        self.h = C.c_void_p()
        check(get_lib().bbg_batch_create(C.byref(self.h)), "bbg_batch_create")

    def close(self):
        if self.h:
            get_lib().bbg_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, integrators, spp, seeds=None):
        n = len(integrators)
        seeds = [it.scene.seed for it in integrators] if seeds is None else seeds
        ints = (C.c_void_p * n)(*[it.h.value for it in integrators])
        cams = (abi.Camera * n)(*[camera(it.scene.camera) for it in integrators])
        params = (abi.RenderParams * n)()
        for i in range(n):
            params[i].spp = spp
            params[i].seed = seeds[i]
        out = abi.Tuning()
        check(get_lib().bbg_batch_autotune(self.h, n, ints, cams, params, C.byref(out)), "bbg_batch_autotune")
        return out

    def render(self, integrators, spp, seeds=None, wave_paths=0, use_graph=True, path_L=False, guides=None,
               train=False, batch=0, lr=0.0, select=0.0, steps=0):
        """Render each GpuPathIntegrator's scene (its own camera) at spp ->
        (list of Film, batch RenderStats). guides: one GpuGuide per scene
        (grouped forward in the batch; trained online with train=True)."""
        n = len(integrators)
        seeds = [it.scene.seed for it in integrators] if seeds is None else seeds
        ints = (C.c_void_p * n)(*[it.h.value for it in integrators])
        cams = (abi.Camera * n)(*[camera(it.scene.camera) for it in integrators])
        params = (abi.RenderParams * n)()
        films, fstructs = [], (abi.Film * n)()
        spps = [spp] * n if isinstance(spp, int) else list(spp)
        for i, it in enumerate(integrators):
            params[i].spp = spps[i]
            params[i].seed = seeds[i]
            params[i].wave_paths = wave_paths
            params[i].use_graph = 1 if use_graph else 0
            if guides is not None:
                params[i].guide = guides[i].h
                params[i].guide_train = 1 if train else 0
                params[i].guide_batch = batch
                params[i].guide_lr = lr
                params[i].guide_select = select
                params[i].guide_steps = steps
            film = Film(cams[i].width, cams[i].height, spps[i], path_L=path_L)
            films.append(film)
            fstructs[i] = film.struct()
        stats = abi.RenderStats()
        check(get_lib().bbg_batch_render(self.h, n, ints, cams, params, fstructs, abi.BBG_MEM_HOST, C.byref(stats)),
              "bbg_batch_render")
        return films, stats


def bsdf_probe(material, wo, wi, u, front_face=True):
    """bbg_bsdf_probe: (n, 12) per query — f rgb, pdf, sample f rgb, wi, pdf, flags (-1: no sample)."""
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    out = np.zeros((wo.shape[0], 12), np.float32)
    check(get_lib().bbg_bsdf_probe(C.byref(material), 1 if front_face else 0, wo.shape[0], _p(wo), _p(wi), _p(u),
                                   _p(out)), "bbg_bsdf_probe")
    return out


def ggx_energy_tables():
    """bbg_ggx_energy_tables: (E 32x32 indexed [alpha][cos], E_avg 32)."""
    e = np.zeros(32 * 32, np.float32)
    a = np.zeros(32, np.float32)
    check(get_lib().bbg_ggx_energy_tables(_p(e), _p(a)), "bbg_ggx_energy_tables")
    return e.reshape(32, 32), a


def dielectric_energy_tables():
    """bbg_dielectric_energy_tables: (E, E_inv) 32x32x32 indexed [alpha][cos][f0]
    and (E_avg, E_inv_avg) 32x32 indexed [alpha][f0]."""
    e = np.zeros(32 ** 3, np.float32)
    ei = np.zeros(32 ** 3, np.float32)
    a = np.zeros(32 * 32, np.float32)
    ai = np.zeros(32 * 32, np.float32)
    check(get_lib().bbg_dielectric_energy_tables(_p(e), _p(ei), _p(a), _p(ai)), "bbg_dielectric_energy_tables")
    return e.reshape(32, 32, 32), ei.reshape(32, 32, 32), a.reshape(32, 32), ai.reshape(32, 32)


def mixture_sample(outputs, u):
    """Sample the vMF mixtures that network output rows (n, 40) describe, with
    uniforms u (n, 3) -> (unit directions (n, 3), mixture density (n,))."""
    outputs = np.ascontiguousarray(outputs, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    n = outputs.shape[0]
    d = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    check(get_lib().bbg_guide_mixture_sample(_p(outputs), _p(u), n, _p(d), _p(pdf)), "bbg_guide_mixture_sample")
    return d, pdf


def mixture_pdf(outputs, dirs):
    """Density of the mixtures (n, 40) at unit directions (n, 3)."""
    outputs = np.ascontiguousarray(outputs, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    pdf = np.zeros(outputs.shape[0], np.float32)
    check(get_lib().bbg_guide_mixture_pdf(_p(outputs), _p(dirs), outputs.shape[0], _p(pdf)), "bbg_guide_mixture_pdf")
    return pdf
