// Oracle harness: the reference renderer (Sopiro/Bulbit, compiled from its own
// sources by oracle/Makefile) behind a small C ABI, so that tests can build the
// same scene on both sides and compare.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product loads this library; only
// tests/, the smoke check and the CPU-baseline leg of bench.py do.
//
// Scenes arrive in the product's own description (include/bbg.h) and are
// built with the reference's public Scene API exactly as a library user would
// (README "Bulbit as a standalone library"): one Mesh for all triangles, one
// Triangle shape + Primitive per triangle (cli/primitive_builder.cpp:63-78),
// Sphere shapes, constant-texture materials, lights in list order, then
// BVH(scene.GetPrimitives()) and PathIntegrator. Private reference state (BVH
// nodes, Mesh arrays, camera basis) is read with a standard-conforming
// member-pointer accessor; the reference sources are not modified.

#include "bbg.h"

#include "bulbit/bulbit.h"
#include "bulbit/bvh.h"
#include "bulbit/cameras.h"
#include "bulbit/integrators.h"
#include "bulbit/lights.h"
#include "bulbit/materials.h"
#include "bulbit/microfacet.h"
#include "bulbit/textures.h"
#include "bulbit/textures3d.h"
#include "bulbit/bxdfs.h"
#include "bulbit/parallel_for.h"
#include "bulbit/samplers.h"
#include "bulbit/scene.h"
#include "bulbit/shapes.h"

#include <chrono>
#include <filesystem>
#include <unordered_map>

using namespace bulbit;

// --- private member access by explicit instantiation --------------------------
// An explicit instantiation may name private members; the friend function it
// defines hands the member pointer out without naming the private type.
template <typename Tag, auto Member>
struct Steal
{
    friend constexpr auto Get(Tag) { return Member; }
};

#define BBREF_STEAL(TAG, MEMBER)                                                                                       \
    struct TAG                                                                                                         \
    {                                                                                                                  \
        friend constexpr auto Get(TAG);                                                                                \
    };                                                                                                                 \
    template struct Steal<TAG, MEMBER>;

BBREF_STEAL(BVHNodes, &BVH::nodes)
BBREF_STEAL(BVHPrims, &BVH::primitives)
BBREF_STEAL(MeshPositions, &Mesh::positions)
BBREF_STEAL(MeshNormals, &Mesh::normals)
BBREF_STEAL(MeshTangents, &Mesh::tangents)
BBREF_STEAL(MeshUVs, &Mesh::texCoords)
BBREF_STEAL(CamOrigin, &PerspectiveCamera::origin)
BBREF_STEAL(CamLowerLeft, &PerspectiveCamera::lower_left)
BBREF_STEAL(CamHorizontal, &PerspectiveCamera::horizontal)
BBREF_STEAL(CamVertical, &PerspectiveCamera::vertical)
BBREF_STEAL(CamU, &PerspectiveCamera::u)
BBREF_STEAL(CamV, &PerspectiveCamera::v)
BBREF_STEAL(CamLensRadius, &PerspectiveCamera::lens_radius)
BBREF_STEAL(GgxE, &TrowbridgeReitzDistribution::E_texture)
BBREF_STEAL(GgxEAvg, &TrowbridgeReitzDistribution::E_avg_texture)
BBREF_STEAL(FloatTexImage, &ImageTexture<Float>::image)
BBREF_STEAL(DmsE, &DielectricMultiScatteringBxDF::E_texture)
BBREF_STEAL(DmsEInv, &DielectricMultiScatteringBxDF::E_inv_texture)
BBREF_STEAL(DmsEAvg, &DielectricMultiScatteringBxDF::E_avg_texture)
BBREF_STEAL(DmsEInvAvg, &DielectricMultiScatteringBxDF::E_inv_avg_texture)
BBREF_STEAL(FloatTex3DImage, &ImageTexture3D<Float>::image)

namespace
{

struct RefScene
{
    Scene scene;
    Mesh* mesh = nullptr;
    std::vector<Light*> lights;
    std::unique_ptr<BVH> bvh;
    std::unique_ptr<PathIntegrator> integrator;
    std::unordered_map<const Primitive*, int32> prim_index;
    int32 n_prims = 0;
};

std::unique_ptr<Filter> MakeFilter(const bbg_camera_spec& s)
{
    switch (s.filter_type)
    {
    case BBG_FILTER_TENT:
        return std::make_unique<TentFilter>(s.filter_extent);
    case BBG_FILTER_GAUSSIAN:
        return std::make_unique<GaussianFilter>(s.filter_sigma, s.filter_extent);
    default:
        return std::make_unique<BoxFilter>(s.filter_extent);
    }
}

struct RefCamera
{
    std::unique_ptr<Filter> filter;
    PerspectiveCamera camera;

    RefCamera(const bbg_camera_spec& s)
        : filter(MakeFilter(s))
        , camera(Transform::LookAt(Point3(s.position[0], s.position[1], s.position[2]),
                                   Point3(s.target[0], s.target[1], s.target[2]), Vec3(s.up[0], s.up[1], s.up[2])),
                 s.vfov_deg, s.aperture_radius, s.focus_distance, Point2i(s.width, s.height), nullptr, filter.get())
    {
    }
};

// The sampler the next integrator and path traces use: IndependentSampler, or
// StratifiedSampler(x_samples, spp / x_samples, jitter, seed).
struct SamplerChoice
{
    int32_t kind = BBG_SAMPLER_INDEPENDENT;
    int32_t x_samples = 1;
    int32_t jitter = 1;
};
SamplerChoice g_sampler;

Sampler* NewSampler(int32_t spp, int32_t seed)
{
    if (g_sampler.kind == BBG_SAMPLER_STRATIFIED)
    {
        return new StratifiedSampler(g_sampler.x_samples, spp / g_sampler.x_samples, g_sampler.jitter != 0, seed);
    }
    return new IndependentSampler(spp, seed);
}

void EnsurePool(int32 threads)
{
    if (threads <= 0)
    {
        threads = int32(std::thread::hardware_concurrency());
    }
    ThreadPool* pool = ThreadPool::global_thread_pool.get();
    if (!pool || pool->WorkerCount() != std::max(threads, 2))
    {
        ThreadPool::global_thread_pool = std::make_unique<ThreadPool>(threads);
    }
}

Spectrum Spec(const float* v)
{
    return Spectrum(v[0], v[1], v[2]);
}

const SpectrumTexture* SpecTex(Scene& scene, const float* v)
{
    return scene.CreateTexture<ConstantTexture, Spectrum>(Spec(v));
}

const FloatTexture* FloatTex(Scene& scene, float v)
{
    return scene.CreateTexture<ConstantTexture, Float>(v);
}

Material* MakeMaterial(Scene& scene, const bbg_material& m)
{
    switch (m.type)
    {
    case BBG_MAT_DIFFUSE:
        return scene.CreateMaterial<DiffuseMaterial>(SpecTex(scene, m.reflectance));
    case BBG_MAT_CONDUCTOR:
        if (m.conductor_from_r)
        {
            return scene.CreateMaterial<ConductorMaterial>(SpecTex(scene, m.k), FloatTex(scene, m.roughness[0]),
                                                           FloatTex(scene, m.roughness[1]),
                                                           SpecTex(scene, m.reflectance), m.energy_compensation != 0);
        }
        return scene.CreateMaterial<ConductorMaterial>(SpecTex(scene, m.eta), SpecTex(scene, m.k),
                                                       FloatTex(scene, m.roughness[0]),
                                                       FloatTex(scene, m.roughness[1]), SpecTex(scene, m.reflectance),
                                                       m.energy_compensation != 0);
    case BBG_MAT_DIELECTRIC:
        return scene.CreateMaterial<DielectricMaterial>(m.eta[0], FloatTex(scene, m.roughness[0]),
                                                        FloatTex(scene, m.roughness[1]), SpecTex(scene, m.reflectance),
                                                        m.energy_compensation != 0);
    case BBG_MAT_METALLIC_ROUGHNESS:
        return scene.CreateMaterial<MetallicRoughnessMaterial>(SpecTex(scene, m.reflectance),
                                                               FloatTex(scene, m.metallic),
                                                               FloatTex(scene, m.roughness[0]),
                                                               FloatTex(scene, m.roughness[1]));
    default:
        return nullptr;
    }
}

// Runs fn with the working directory set to a scratch folder: the reference's
// Integrator constructor creates "res/refs" relative to the working directory
// (src/bxdf/microfacet.cpp:14,241).
template <typename F>
void InScratchDir(F&& fn)
{
    namespace fs = std::filesystem;
    fs::path old = fs::current_path();
    fs::path scratch = fs::temp_directory_path() / "bbref_scratch";
    fs::create_directories(scratch);
    fs::current_path(scratch);
    fn();
    fs::current_path(old);
}

} // namespace

extern "C" {

int bbref_init(int32_t threads)
{
    EnsurePool(threads);
    return ThreadPool::global_thread_pool->WorkerCount();
}

// Builds the reference scene and its BVH (timed; seconds in *build_seconds).
void* bbref_scene_create(const bbg_geometry* g, const int32_t* prim_material, const bbg_material* materials,
                         int32_t n_materials, const bbg_light* lights, int32_t n_lights, double* build_seconds)
{
    EnsurePool(0);
    auto* rs = new RefScene;
    Scene& scene = rs->scene;

    if (g->n_triangles > 0)
    {
        std::vector<Point3> pos(g->n_vertices);
        std::vector<Vec3> nrm(g->n_vertices), tan(g->n_vertices);
        std::vector<Point2> uv(g->n_vertices);
        for (int32 i = 0; i < g->n_vertices; ++i)
        {
            pos[i] = Point3(g->positions[3 * i], g->positions[3 * i + 1], g->positions[3 * i + 2]);
            nrm[i] = g->normals ? Vec3(g->normals[3 * i], g->normals[3 * i + 1], g->normals[3 * i + 2]) : z_axis;
            tan[i] = g->tangents ? Vec3(g->tangents[3 * i], g->tangents[3 * i + 1], g->tangents[3 * i + 2]) : x_axis;
            uv[i] = g->uvs ? Point2(g->uvs[2 * i], g->uvs[2 * i + 1]) : Point2(0, 0);
        }
        std::vector<int32> idx(g->tri_indices, g->tri_indices + 3 * size_t(g->n_triangles));
        rs->mesh = scene.CreateMesh(std::move(pos), std::move(nrm), std::move(tan), std::move(uv), std::move(idx),
                                    Mat4(identity));
    }

    std::vector<Material*> mats(n_materials);
    for (int32 i = 0; i < n_materials; ++i)
    {
        mats[i] = MakeMaterial(scene, materials[i]);
    }

    rs->n_prims = g->n_prims;
    for (int32 i = 0; i < g->n_prims; ++i)
    {
        Shape* shape;
        if (g->prim_kind[i] == BBG_PRIM_TRIANGLE)
        {
            shape = scene.CreateShape<Triangle>(rs->mesh, size_t(g->prim_index[i]));
        }
        else
        {
            const bbg_sphere& s = g->spheres[g->prim_index[i]];
            Transform tf(Vec3(s.p[0], s.p[1], s.p[2]), Quat(s.q[0], s.q[1], s.q[2], s.q[3]),
                         Vec3(s.s[0], s.s[1], s.s[2]));
            shape = scene.CreateShape<Sphere>(tf, s.radius);
        }
        int32 m = prim_material ? prim_material[i] : -1;
        Primitive* p = scene.CreatePrimitive(shape, m >= 0 ? mats[m] : nullptr, MediumInterface{});
        rs->prim_index[p] = i;
    }

    const std::vector<Primitive*>& prims = scene.GetPrimitives();
    for (int32 i = 0; i < n_lights; ++i)
    {
        const bbg_light& l = lights[i];
        Light* light = nullptr;
        switch (l.type)
        {
        case BBG_LIGHT_POINT:
            light = scene.CreateLight<PointLight>(Point3(l.position[0], l.position[1], l.position[2]),
                                                  Spec(l.intensity), nullptr);
            break;
        case BBG_LIGHT_SPOT:
            light = scene.CreateLight<SpotLight>(Point3(l.position[0], l.position[1], l.position[2]),
                                                 Vec3(l.direction[0], l.direction[1], l.direction[2]),
                                                 Spec(l.intensity), l.angle_max, l.angle_falloff_start, nullptr);
            break;
        case BBG_LIGHT_UNIFORM_INFINITE:
            light = scene.CreateLight<UniformInfiniteLight>(Spec(l.intensity), l.scale);
            break;
        case BBG_LIGHT_DIFFUSE_AREA:
            light = scene.CreateLight<DiffuseAreaLight>(prims[l.prim], SpecTex(scene, l.intensity), l.two_sided != 0);
            break;
        }
        rs->lights.push_back(light);
    }

    auto t0 = std::chrono::steady_clock::now();
    rs->bvh = std::make_unique<BVH>(scene.GetPrimitives());
    auto t1 = std::chrono::steady_clock::now();
    if (build_seconds)
    {
        *build_seconds = std::chrono::duration<double>(t1 - t0).count();
    }
    return rs;
}

void bbref_scene_destroy(void* handle)
{
    // BVH::~BVH deletes its node array with the wrong form of delete
    // (src/accel/bvh.cpp:53); leak the tree rather than trip over that.
    auto* rs = static_cast<RefScene*>(handle);
    (void)rs->bvh.release();
    delete rs;
}

// Creates the PathIntegrator (timed: the constructor precomputes reflectance
// tables, src/integrator/integrator.cpp:151).
int bbref_integrator_create(void* handle, int32_t spp, int32_t seed, int32_t max_bounces, int32_t rr_min_bounces,
                            int32_t regularize, double* seconds)
{
    auto* rs = static_cast<RefScene*>(handle);
    Sampler* sampler = NewSampler(spp, seed); // owned for the process lifetime (non-owning in the API)
    auto t0 = std::chrono::steady_clock::now();
    InScratchDir([&] {
        rs->integrator = std::make_unique<PathIntegrator>(rs->bvh.get(), rs->lights, sampler, max_bounces,
                                                          rr_min_bounces, regularize != 0);
    });
    auto t1 = std::chrono::steady_clock::now();
    if (seconds)
    {
        *seconds = std::chrono::duration<double>(t1 - t0).count();
    }
    return 0;
}

int32_t bbref_bvh_node_count(void* handle)
{
    auto* rs = static_cast<RefScene*>(handle);
    const auto* nodes = rs->bvh.get()->*Get(BVHNodes{});
    // Count nodes reachable from the root (the flattened array is dense).
    int32 count = 0;
    std::vector<int32> stack{ 0 };
    while (!stack.empty())
    {
        int32 i = stack.back();
        stack.pop_back();
        ++count;
        if (nodes[i].primitive_count == 0)
        {
            stack.push_back(i + 1);
            stack.push_back(nodes[i].child2_offset);
        }
    }
    return count;
}

// The reference's flattened tree, node for node, and per leaf slot the
// primitive's index in scene.GetPrimitives().
int bbref_bvh_export(void* handle, bbg_bvh_node* nodes_out, int32_t* slot_prims_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    const auto* nodes = rs->bvh.get()->*Get(BVHNodes{});
    const auto& prims = rs->bvh.get()->*Get(BVHPrims{});
    int32 n = bbref_bvh_node_count(handle);
    for (int32 i = 0; i < n; ++i)
    {
        bbg_bvh_node& o = nodes_out[i];
        std::memset(&o, 0, sizeof(o));
        o.bmin[0] = nodes[i].aabb.min.x;
        o.bmin[1] = nodes[i].aabb.min.y;
        o.bmin[2] = nodes[i].aabb.min.z;
        o.bmax[0] = nodes[i].aabb.max.x;
        o.bmax[1] = nodes[i].aabb.max.y;
        o.bmax[2] = nodes[i].aabb.max.z;
        o.offset = nodes[i].primitives_offset;
        o.count = nodes[i].primitive_count;
        o.axis = nodes[i].primitive_count == 0 ? nodes[i].axis : 0;
    }
    for (size_t i = 0; i < prims.size(); ++i)
    {
        slot_prims_out[i] = rs->prim_index.at(prims[i]);
    }
    return n;
}

// The reference Mesh's world-space arrays after construction (Mesh::Mesh
// re-normalises normals and tangents, src/geometry/mesh.cpp:23-33).
int bbref_mesh_export(void* handle, float* positions, float* normals, float* tangents, float* uvs)
{
    auto* rs = static_cast<RefScene*>(handle);
    if (!rs->mesh)
    {
        return 0;
    }
    const auto& p = rs->mesh->*Get(MeshPositions{});
    const auto& n = rs->mesh->*Get(MeshNormals{});
    const auto& t = rs->mesh->*Get(MeshTangents{});
    const auto& uv = rs->mesh->*Get(MeshUVs{});
    for (size_t i = 0; i < p.size(); ++i)
    {
        for (int k = 0; k < 3; ++k)
        {
            if (positions) positions[3 * i + k] = p[i][k];
            if (normals) normals[3 * i + k] = n[i][k];
            if (tangents) tangents[3 * i + k] = t[i][k];
        }
        if (uvs)
        {
            uvs[2 * i] = uv[i].x;
            uvs[2 * i + 1] = uv[i].y;
        }
    }
    return int(p.size());
}

// Batched BVH::Intersect over C threads (ParallelFor), the CPU baseline of the
// ray microbenchmark. Returns wall seconds.
double bbref_intersect(void* handle, const bbg_ray* rays, int64_t n, bbg_hit* hits)
{
    auto* rs = static_cast<RefScene*>(handle);
    const BVH* bvh = rs->bvh.get();
    auto t0 = std::chrono::steady_clock::now();
    ParallelFor(0, int32(n), [&](int32 b, int32 e) {
        for (int32 i = b; i < e; ++i)
        {
            const bbg_ray& r = rays[i];
            Ray ray(Point3(r.o[0], r.o[1], r.o[2]), Vec3(r.d[0], r.d[1], r.d[2]));
            Intersection isect;
            if (bvh->Intersect(&isect, ray, r.t_min, r.t_max))
            {
                hits[i].prim = rs->prim_index.at(isect.primitive);
                hits[i].t = isect.t;
            }
            else
            {
                hits[i].prim = -1;
                hits[i].t = r.t_max;
            }
            hits[i].u = 0;
            hits[i].v = 0;
        }
    });
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Batched BVH::IntersectAny. Returns wall seconds.
double bbref_intersect_any(void* handle, const bbg_ray* rays, int64_t n, uint8_t* occluded)
{
    auto* rs = static_cast<RefScene*>(handle);
    const BVH* bvh = rs->bvh.get();
    auto t0 = std::chrono::steady_clock::now();
    ParallelFor(0, int32(n), [&](int32 b, int32 e) {
        for (int32 i = b; i < e; ++i)
        {
            const bbg_ray& r = rays[i];
            Ray ray(Point3(r.o[0], r.o[1], r.o[2]), Vec3(r.d[0], r.d[1], r.d[2]));
            occluded[i] = bvh->IntersectAny(ray, r.t_min, r.t_max) ? 1 : 0;
        }
    });
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Every primitive hit by one ray in [t_min, t_max] (brute force over the
// primitive list): used to find near-ties between the two nearest hits.
int bbref_intersect_all(void* handle, const bbg_ray* r, int32_t max_out, int32_t* prims_out, float* t_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    const auto& prims = rs->scene.GetPrimitives();
    Ray ray(Point3(r->o[0], r->o[1], r->o[2]), Vec3(r->d[0], r->d[1], r->d[2]));
    int count = 0;
    for (size_t i = 0; i < prims.size(); ++i)
    {
        Intersection isect;
        if (prims[i]->Intersect(&isect, ray, r->t_min, r->t_max))
        {
            if (count < max_out)
            {
                prims_out[count] = int32(i);
                t_out[count] = isect.t;
            }
            ++count;
        }
    }
    return count;
}

// Traversal work of BVH::RayCast (include/bulbit/bvh.h:102-155) for each
// query: its loop replayed with the reference's own nodes, AABB::TestRay and
// Primitive::Intersect / IntersectAny, counting nodes popped (each is
// slab-tested) and primitive tests, for closest-hit (any = 0, the
// BVH::Intersect callback) or any-hit (the BVH::IntersectAny callback)
// queries. Returns the totals over the n rays.
int bbref_count_traversal(void* handle, const bbg_ray* rays, int64_t n, int32_t any, int64_t* nodes_out,
                          int64_t* prims_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    const auto* nodes = rs->bvh.get()->*Get(BVHNodes{});
    const auto& prims = rs->bvh.get()->*Get(BVHPrims{});
    int64_t total_nodes = 0, total_prims = 0;
    for (int64_t k = 0; k < n; ++k)
    {
        const bbg_ray& br = rays[k];
        Ray r(Point3(br.o[0], br.o[1], br.o[2]), Vec3(br.d[0], br.d[1], br.d[2]));
        Float t_min = br.t_min, t_max = br.t_max;
        const Vec3 inv_dir(1 / r.d.x, 1 / r.d.y, 1 / r.d.z);
        const int32 is_dir_neg[3] = { int32(inv_dir.x < 0), int32(inv_dir.y < 0), int32(inv_dir.z < 0) };
        std::vector<int32> stack{ 0 };
        bool done = false;
        while (!stack.empty() && !done)
        {
            int32 index = stack.back();
            stack.pop_back();
            ++total_nodes;
            if (!nodes[index].aabb.TestRay(r.o, t_min, t_max, inv_dir, is_dir_neg))
            {
                continue;
            }
            if (nodes[index].primitive_count > 0)
            {
                for (int32 i = 0; i < nodes[index].primitive_count; ++i)
                {
                    ++total_prims;
                    const Primitive* p = prims[nodes[index].primitives_offset + i];
                    Float t;
                    if (any)
                    {
                        t = p->IntersectAny(r, t_min, t_max) ? t_min : t_max;
                    }
                    else
                    {
                        Intersection isect;
                        t = p->Intersect(&isect, r, t_min, t_max) ? isect.t : t_max;
                    }
                    if (t <= t_min)
                    {
                        done = true;
                        break;
                    }
                    t_max = t;
                }
            }
            else
            {
                int32 child1 = index + 1;
                int32 child2 = nodes[index].child2_offset;
                if (is_dir_neg[nodes[index].axis])
                {
                    stack.push_back(child1);
                    stack.push_back(child2);
                }
                else
                {
                    stack.push_back(child2);
                    stack.push_back(child1);
                }
            }
        }
    }
    *nodes_out = total_nodes;
    *prims_out = total_prims;
    return 0;
}

// Material::GetBSDF at a surface with shading normal +z and tangent +x, then
// BSDF::f, PDF and Sample_f per query, in bbg_bsdf_probe's output layout.
int bbref_bsdf_probe(const bbg_material* m, int32_t front_face, int32_t n, const float* wo, const float* wi,
                     const float* u, float* out)
{
    EnsurePool(0);
    static bool tables = false;
    if (!tables)
    {
        InScratchDir([] { PrepareReflectanceTextures(32, 1024); });
        tables = true;
    }
    Scene scene;
    const Material* mat = MakeMaterial(scene, *m);
    Intersection isect{};
    isect.front_face = front_face != 0;
    isect.normal = Vec3(0, 0, 1);
    isect.shading.normal = Vec3(0, 0, 1);
    isect.shading.tangent = Vec3(1, 0, 0);
    isect.uv = Point2(0.5f, 0.5f);
    Allocator alloc;
    BSDF bsdf;
    if (!mat || !mat->GetBSDF(&bsdf, isect, alloc))
    {
        return -1;
    }
    for (int32_t i = 0; i < n; ++i)
    {
        Vec3 o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        Vec3 w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        Spectrum f = bsdf.f(o, w);
        Float pdf = bsdf.PDF(o, w);
        BSDFSample s;
        bool ok = bsdf.Sample_f(&s, o, u[3 * i], Point2(u[3 * i + 1], u[3 * i + 2]));
        float* r = out + 12 * size_t(i);
        r[0] = f.r, r[1] = f.g, r[2] = f.b, r[3] = pdf;
        r[4] = ok ? s.f.r : 0, r[5] = ok ? s.f.g : 0, r[6] = ok ? s.f.b : 0;
        r[7] = ok ? s.wi.x : 0, r[8] = ok ? s.wi.y : 0, r[9] = ok ? s.wi.z : 0;
        r[10] = ok ? s.pdf : 0, r[11] = ok ? float(int32(s.flags)) : -1.0f;
    }
    return 0;
}

// The derived state of the reference PerspectiveCamera for a spec.
int bbref_camera(const bbg_camera_spec* spec, bbg_camera* out)
{
    RefCamera rc(*spec);
    const PerspectiveCamera& c = rc.camera;
    auto put = [](float* dst, const Vec3& v) {
        dst[0] = v.x;
        dst[1] = v.y;
        dst[2] = v.z;
    };
    out->width = spec->width;
    out->height = spec->height;
    put(out->origin, c.*Get(CamOrigin{}));
    put(out->lower_left, c.*Get(CamLowerLeft{}));
    put(out->horizontal, c.*Get(CamHorizontal{}));
    put(out->vertical, c.*Get(CamVertical{}));
    put(out->u, c.*Get(CamU{}));
    put(out->v, c.*Get(CamV{}));
    out->lens_radius = c.*Get(CamLensRadius{});
    out->filter_extent = spec->filter_extent;
    out->filter_type = spec->filter_type;
    out->filter_sigma = spec->filter_sigma;
    return 0;
}

// Per-path radiance: for each requested path (index (y*W + x)*spp + sample)
// the body of UniDirectionalRayIntegrator::Render's inner loop
// (src/integrator/integrator.cpp:185-192), including its argument evaluation
// order, then PathIntegrator::Li. L_out gets 3 floats per requested path.
// path_ids == NULL means every path of the image. Returns wall seconds.
double bbref_trace_paths(void* handle, const bbg_camera_spec* spec, int32_t spp, int32_t seed, const int64_t* path_ids,
                         int64_t n, float* L_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    RefCamera rc(*spec);
    const Camera* camera = &rc.camera;
    const PathIntegrator* integrator = rs->integrator.get();
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<Sampler> proto(NewSampler(spp, seed));
    ParallelFor(0, int32(n), [&](int32 b, int32 e) {
        int8 mem[128];
        BufferResource buffer(mem, sizeof(mem));
        Allocator alloc(&buffer);
        Sampler* sampler = proto->Clone(alloc);
        for (int32 i = b; i < e; ++i)
        {
            int64 id = path_ids ? path_ids[i] : i;
            int32 sample = int32(id % spp);
            int64 pixel_index = id / spp;
            Point2i pixel(int32(pixel_index % spec->width), int32(pixel_index / spec->width));

            sampler->StartPixelSample(pixel, sample);

            PrimaryRay primary_ray;
            camera->SampleRay(&primary_ray, pixel, sampler->Next2D(), sampler->Next2D());

            Spectrum L = integrator->Li(primary_ray.ray, camera->GetMedium(), *sampler);
            L_out[3 * i] = L.r;
            L_out[3 * i + 1] = L.g;
            L_out[3 * i + 2] = L.b;
        }
    });
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// The reference render itself: Render() then Rendering::Wait() (the caller
// joins the pool), timed. image_out gets Film::GetRenderedImage (3 floats per
// pixel) and variance_out, if not NULL, Film::GetVarianceImage. Returns wall
// seconds of Render + Wait.
double bbref_render(void* handle, const bbg_camera_spec* spec, float* image_out, float* variance_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    RefCamera rc(*spec);
    Allocator alloc;
    auto t0 = std::chrono::steady_clock::now();
    Rendering* rendering = rs->integrator->Render(alloc, &rc.camera);
    rendering->Wait();
    auto t1 = std::chrono::steady_clock::now();
    const Film& film = rendering->GetFilm();
    Image3 image = film.GetRenderedImage();
    for (int32 i = 0; i < image.width * image.height; ++i)
    {
        image_out[3 * i] = image[i].r;
        image_out[3 * i + 1] = image[i].g;
        image_out[3 * i + 2] = image[i].b;
    }
    if (variance_out)
    {
        Image1 var = film.GetVarianceImage();
        for (int32 i = 0; i < var.width * var.height; ++i)
        {
            variance_out[i] = var[i];
        }
    }
    alloc.delete_object(rendering);
    return std::chrono::duration<double>(t1 - t0).count();
}

// PowerLightSampler pmf of each light, in list order.
int bbref_light_pmf(void* handle, float* pmf_out)
{
    auto* rs = static_cast<RefScene*>(handle);
    const LightSampler* ls = rs->integrator->GetLightSampler();
    for (size_t i = 0; i < rs->lights.size(); ++i)
    {
        pmf_out[i] = ls->EvaluatePMF(rs->lights[i]);
    }
    return int(rs->lights.size());
}

// The first n draws of IndependentSampler after StartPixelSample.
void bbref_set_sampler(int32_t kind, int32_t x_samples, int32_t jitter)
{
    g_sampler = SamplerChoice{ kind, x_samples, jitter };
}

// The reference's GGX energy tables after PrepareReflectanceTextures(32, 1024)
// (what every Integrator constructor runs): E 32 x 32, E_avg 32.
int bbref_ggx_energy_tables(float* e_out, float* e_avg_out)
{
    EnsurePool(0);
    InScratchDir([] { PrepareReflectanceTextures(32, 1024); });
    const auto& e = *(*Get(GgxE{}));
    const auto& e_avg = *(*Get(GgxEAvg{}));
    const auto& ei = e.*Get(FloatTexImage{});
    const auto& ai = e_avg.*Get(FloatTexImage{});
    for (int32 i = 0; i < 32 * 32; ++i)
    {
        e_out[i] = ei[i];
    }
    for (int32 i = 0; i < 32; ++i)
    {
        e_avg_out[i] = ai[i];
    }
    return 0;
}

// The reference's rough-dielectric energy tables after
// PrepareReflectanceTextures(32, 1024): E, E_inv 32^3 and E_avg, E_inv_avg 32^2
// in the images' own layouts.
int bbref_dielectric_energy_tables(float* e_out, float* e_inv_out, float* e_avg_out, float* e_inv_avg_out)
{
    EnsurePool(0);
    InScratchDir([] { PrepareReflectanceTextures(32, 1024); });
    const auto& e = (*(*Get(DmsE{}))).*Get(FloatTex3DImage{});
    const auto& ei = (*(*Get(DmsEInv{}))).*Get(FloatTex3DImage{});
    const auto& a = (*(*Get(DmsEAvg{}))).*Get(FloatTexImage{});
    const auto& ai = (*(*Get(DmsEInvAvg{}))).*Get(FloatTexImage{});
    for (int32 i = 0; i < 32 * 32 * 32; ++i)
    {
        e_out[i] = e[i];
        e_inv_out[i] = ei[i];
    }
    for (int32 i = 0; i < 32 * 32; ++i)
    {
        e_avg_out[i] = a[i];
        e_inv_avg_out[i] = ai[i];
    }
    return 0;
}

int bbref_sampler_draws(int32_t px, int32_t py, int32_t seed, int32_t sample, int32_t n, float* out)
{
    IndependentSampler s(1, seed);
    s.StartPixelSample(Point2i(px, py), sample);
    for (int32 i = 0; i < n; ++i)
    {
        out[i] = s.Next1D();
    }
    return n;
}

// Raw PCG32 output after RNG(initstate, initseq) (include/bulbit/random.h:21).
int bbref_pcg32(uint64_t initstate, uint64_t initseq, int32_t n, uint32_t* out)
{
    RNG rng(initstate, initseq);
    for (int32 i = 0; i < n; ++i)
    {
        out[i] = rng.NextUint();
    }
    return n;
}

uint64_t bbref_hash_pixel_sample(int32_t px, int32_t py, int32_t seed, int32_t sample)
{
    return Hash(Point2i(px, py), seed, sample);
}

} // extern "C"
