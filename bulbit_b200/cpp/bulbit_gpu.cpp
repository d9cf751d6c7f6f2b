// The C++ drop-in classes of include/bulbit_gpu.hpp: the reference's scene
// objects translated once into the C ABI's plain arrays (bbg.h), then every
// query and render runs in libbulbit_b200.so.
//
// Private reference state (BVH nodes, Mesh arrays, Triangle vertex indices,
// camera basis, light and material parameters, constant-texture values) is
// read through a standard-conforming accessor: an explicit instantiation may
// name a private member, and the friend function it defines returns the
// member pointer. The reference sources are used unmodified.

#include "bulbit_gpu.hpp"

#include "bulbit/parallel_for.h"
#include "bulbit/textures.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

namespace
{

template <typename Tag, auto Member>
struct Steal
{
    friend constexpr auto Get(Tag) { return Member; }
};

#define BULBIT_GPU_STEAL(TAG, MEMBER)                                                                                  \
    struct TAG                                                                                                         \
    {                                                                                                                  \
        friend constexpr auto Get(TAG);                                                                                \
    };                                                                                                                 \
    template struct Steal<TAG, MEMBER>;

using namespace bulbit;

BULBIT_GPU_STEAL(BvhNodes, &BVH::nodes)
BULBIT_GPU_STEAL(BvhPrims, &BVH::primitives)
BULBIT_GPU_STEAL(TriMesh, &Triangle::mesh)
BULBIT_GPU_STEAL(TriV, &Triangle::v)
BULBIT_GPU_STEAL(MeshPositions, &Mesh::positions)
BULBIT_GPU_STEAL(MeshNormals, &Mesh::normals)
BULBIT_GPU_STEAL(MeshTangents, &Mesh::tangents)
BULBIT_GPU_STEAL(MeshUVs, &Mesh::texCoords)
BULBIT_GPU_STEAL(MeshIndices, &Mesh::indices)
BULBIT_GPU_STEAL(CamOrigin, &PerspectiveCamera::origin)
BULBIT_GPU_STEAL(CamLowerLeft, &PerspectiveCamera::lower_left)
BULBIT_GPU_STEAL(CamHorizontal, &PerspectiveCamera::horizontal)
BULBIT_GPU_STEAL(CamVertical, &PerspectiveCamera::vertical)
BULBIT_GPU_STEAL(CamU, &PerspectiveCamera::u)
BULBIT_GPU_STEAL(CamV, &PerspectiveCamera::v)
BULBIT_GPU_STEAL(CamLensRadius, &PerspectiveCamera::lens_radius)
BULBIT_GPU_STEAL(FilmSamples, &Film::samples)
BULBIT_GPU_STEAL(FilmCounts, &Film::sample_counts)
BULBIT_GPU_STEAL(FilmMoments, &Film::moments)
BULBIT_GPU_STEAL(SamplerSeed, &IndependentSampler::seed)
BULBIT_GPU_STEAL(StratSeed, &StratifiedSampler::seed)
BULBIT_GPU_STEAL(StratX, &StratifiedSampler::x_samples)
BULBIT_GPU_STEAL(StratJitter, &StratifiedSampler::jitter)
BULBIT_GPU_STEAL(ConstSpec, &ConstantTexture<Spectrum>::value)
BULBIT_GPU_STEAL(ConstFloat, &ConstantTexture<Float>::value)
BULBIT_GPU_STEAL(CondEta, &ConductorMaterial::eta)
BULBIT_GPU_STEAL(CondK, &ConductorMaterial::k)
BULBIT_GPU_STEAL(CondU, &ConductorMaterial::u_roughness)
BULBIT_GPU_STEAL(CondV, &ConductorMaterial::v_roughness)
BULBIT_GPU_STEAL(CondRefl, &ConductorMaterial::reflectance)
BULBIT_GPU_STEAL(CondEc, &ConductorMaterial::energy_compensation)
BULBIT_GPU_STEAL(CondNormal, &ConductorMaterial::normal)
BULBIT_GPU_STEAL(CondAlpha, &ConductorMaterial::alpha)
BULBIT_GPU_STEAL(DielEta, &DielectricMaterial::eta)
BULBIT_GPU_STEAL(DielU, &DielectricMaterial::u_roughness)
BULBIT_GPU_STEAL(DielV, &DielectricMaterial::v_roughness)
BULBIT_GPU_STEAL(DielRefl, &DielectricMaterial::reflectance)
BULBIT_GPU_STEAL(DielEc, &DielectricMaterial::energy_compensation)
BULBIT_GPU_STEAL(DielNormal, &DielectricMaterial::normal)
BULBIT_GPU_STEAL(MrBase, &MetallicRoughnessMaterial::basecolor)
BULBIT_GPU_STEAL(MrMetallic, &MetallicRoughnessMaterial::metallic)
BULBIT_GPU_STEAL(MrU, &MetallicRoughnessMaterial::u_roughness)
BULBIT_GPU_STEAL(MrV, &MetallicRoughnessMaterial::v_roughness)
BULBIT_GPU_STEAL(MrNormal, &MetallicRoughnessMaterial::normal)
BULBIT_GPU_STEAL(MrAlpha, &MetallicRoughnessMaterial::alpha)
BULBIT_GPU_STEAL(PointP, &PointLight::p)
BULBIT_GPU_STEAL(PointI, &PointLight::intensity)
BULBIT_GPU_STEAL(SpotP, &SpotLight::p)
BULBIT_GPU_STEAL(SpotFrame, &SpotLight::frame)
BULBIT_GPU_STEAL(SpotCosMin, &SpotLight::cos_theta_min)
BULBIT_GPU_STEAL(SpotCosMax, &SpotLight::cos_theta_max)
BULBIT_GPU_STEAL(SpotI, &SpotLight::intensity)
BULBIT_GPU_STEAL(InfL, &UniformInfiniteLight::l)
BULBIT_GPU_STEAL(InfScale, &UniformInfiniteLight::scale)
BULBIT_GPU_STEAL(AreaEmission, &DiffuseAreaLight::emission)
BULBIT_GPU_STEAL(AreaTwoSided, &DiffuseAreaLight::two_sided)

[[noreturn]] void Unsupported(const std::string& what)
{
    throw std::runtime_error("bulbit_gpu: " + what);
}

void Check(bbg_status s, const char* where)
{
    if (s != BBG_OK)
    {
        throw std::runtime_error(std::string("bulbit_gpu: ") + where + ": " + bbg_last_error());
    }
}

void Put3(float* out, const Vec3& v)
{
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

void PutSpec(float* out, const Spectrum& s)
{
    out[0] = s.r;
    out[1] = s.g;
    out[2] = s.b;
}

Spectrum ConstSpectrum(const SpectrumTexture* t, const char* what)
{
    auto* c = dynamic_cast<const ConstantTexture<Spectrum>*>(t);
    if (!c)
    {
        Unsupported(std::string(what) + ": only constant textures are supported");
    }
    return c->*Get(ConstSpec{});
}

Float ConstScalar(const FloatTexture* t, const char* what)
{
    auto* c = dynamic_cast<const ConstantTexture<Float>*>(t);
    if (!c)
    {
        Unsupported(std::string(what) + ": only constant textures are supported");
    }
    return c->*Get(ConstFloat{});
}

// True when the alpha test never discards a hit: no alpha texture, or a
// constant one that is not below 1 (include/bulbit/primitive.h:60-66 tests
// only alpha < 1), which is what the CLI's material builders attach
// (cli/material_builder.cpp, alpha = 1 by default).
bool OpaqueAlpha(const FloatTexture* alpha)
{
    if (!alpha)
    {
        return true;
    }
    auto* c = dynamic_cast<const ConstantTexture<Float>*>(alpha);
    return c && !(c->*Get(ConstFloat{}) < 1);
}

// The material of one primitive as the device describes it
// (src/material/*_material.cpp GetBSDF, constant textures only).
bbg_material TranslateMaterial(const Material* m)
{
    bbg_material out{};
    if (m->Is<DiffuseMaterial>())
    {
        const DiffuseMaterial* d = m->Cast<DiffuseMaterial>();
        if (d->normal || !OpaqueAlpha(d->alpha))
        {
            Unsupported("DiffuseMaterial with a normal texture or alpha below 1");
        }
        // GetBSDF takes LambertianBxDF unless the roughness is > 0
        // (src/material/diffuse_material.cpp:22-33).
        if (d->roughness && ConstScalar(d->roughness, "DiffuseMaterial roughness") > 0)
        {
            Unsupported("DiffuseMaterial with roughness > 0 (EONBxDF)");
        }
        out.type = BBG_MAT_DIFFUSE;
        PutSpec(out.reflectance, ConstSpectrum(d->reflectance, "DiffuseMaterial reflectance"));
    }
    else if (m->Is<ConductorMaterial>())
    {
        const ConductorMaterial* c = m->Cast<ConductorMaterial>();
        if (c->*Get(CondNormal{}) || !OpaqueAlpha(c->*Get(CondAlpha{})))
        {
            Unsupported("ConductorMaterial with a normal texture or alpha below 1");
        }
        out.type = BBG_MAT_CONDUCTOR;
        const SpectrumTexture* eta = c->*Get(CondEta{});
        out.conductor_from_r = eta ? 0 : 1;
        if (eta)
        {
            PutSpec(out.eta, ConstSpectrum(eta, "ConductorMaterial eta"));
        }
        PutSpec(out.k, ConstSpectrum(c->*Get(CondK{}), "ConductorMaterial k"));
        const SpectrumTexture* refl = c->*Get(CondRefl{});
        PutSpec(out.reflectance, refl ? ConstSpectrum(refl, "ConductorMaterial reflectance") : Spectrum(1));
        out.roughness[0] = ConstScalar(c->*Get(CondU{}), "ConductorMaterial roughness");
        out.roughness[1] = ConstScalar(c->*Get(CondV{}), "ConductorMaterial roughness");
        out.energy_compensation = (c->*Get(CondEc{})) ? 1 : 0;
    }
    else if (m->Is<DielectricMaterial>())
    {
        const DielectricMaterial* d = m->Cast<DielectricMaterial>();
        if (d->*Get(DielNormal{}))
        {
            Unsupported("DielectricMaterial with a normal texture");
        }
        out.type = BBG_MAT_DIELECTRIC;
        Float eta = d->*Get(DielEta{});
        out.eta[0] = out.eta[1] = out.eta[2] = eta;
        const SpectrumTexture* refl = d->*Get(DielRefl{});
        PutSpec(out.reflectance, refl ? ConstSpectrum(refl, "DielectricMaterial reflectance") : Spectrum(1));
        out.roughness[0] = ConstScalar(d->*Get(DielU{}), "DielectricMaterial roughness");
        out.roughness[1] = ConstScalar(d->*Get(DielV{}), "DielectricMaterial roughness");
        out.energy_compensation = (d->*Get(DielEc{})) ? 1 : 0;
    }
    else if (m->Is<MetallicRoughnessMaterial>())
    {
        const MetallicRoughnessMaterial* r = m->Cast<MetallicRoughnessMaterial>();
        if (r->*Get(MrNormal{}) || !OpaqueAlpha(r->*Get(MrAlpha{})))
        {
            Unsupported("MetallicRoughnessMaterial with a normal texture or alpha below 1");
        }
        out.type = BBG_MAT_METALLIC_ROUGHNESS;
        PutSpec(out.reflectance, ConstSpectrum(r->*Get(MrBase{}), "MetallicRoughnessMaterial basecolor"));
        out.metallic = ConstScalar(r->*Get(MrMetallic{}), "MetallicRoughnessMaterial metallic");
        out.roughness[0] = ConstScalar(r->*Get(MrU{}), "MetallicRoughnessMaterial roughness");
        out.roughness[1] = ConstScalar(r->*Get(MrV{}), "MetallicRoughnessMaterial roughness");
    }
    else
    {
        Unsupported("material type " + std::to_string(m->type_index) + " (supported: Diffuse, Conductor, Dielectric, "
                    "MetallicRoughness)");
    }
    return out;
}

// A light after Integrator's Preprocess, in the device description. The
// spot light's cone angles are recovered from its stored cosines.
bbg_light TranslateLight(const Light* l, const bulbit_gpu::GpuBVH& accel)
{
    bbg_light out{};
    out.prim = -1;
    out.scale = 1;
    if (l->Is<PointLight>())
    {
        const PointLight* p = l->Cast<PointLight>();
        out.type = BBG_LIGHT_POINT;
        Put3(out.position, p->*Get(PointP{}));
        PutSpec(out.intensity, p->*Get(PointI{}));
    }
    else if (l->Is<SpotLight>())
    {
        const SpotLight* s = l->Cast<SpotLight>();
        out.type = BBG_LIGHT_SPOT;
        Put3(out.position, s->*Get(SpotP{}));
        const Frame& f = s->*Get(SpotFrame{});
        Put3(out.direction, -f.z); // the constructor stores frame = FromZ(-Normalize(direction))
        PutSpec(out.intensity, s->*Get(SpotI{}));
        const double rad_to_deg = 180.0 / 3.14159265358979323846;
        out.angle_max = float(std::acos(double(s->*Get(SpotCosMax{}))) * rad_to_deg);
        out.angle_falloff_start = float(std::acos(double(s->*Get(SpotCosMin{}))) * rad_to_deg);
    }
    else if (l->Is<UniformInfiniteLight>())
    {
        const UniformInfiniteLight* u = l->Cast<UniformInfiniteLight>();
        out.type = BBG_LIGHT_UNIFORM_INFINITE;
        PutSpec(out.intensity, u->*Get(InfL{}));
        out.scale = u->*Get(InfScale{});
    }
    else if (l->Is<DiffuseAreaLight>())
    {
        const DiffuseAreaLight* a = l->Cast<DiffuseAreaLight>();
        out.type = BBG_LIGHT_DIFFUSE_AREA;
        out.prim = accel.IndexOf(a->primitive);
        if (out.prim < 0)
        {
            Unsupported("area light on a primitive that is not in the accel");
        }
        out.two_sided = (a->*Get(AreaTwoSided{})) ? 1 : 0;
        PutSpec(out.intensity, ConstSpectrum(a->*Get(AreaEmission{}), "DiffuseAreaLight emission"));
    }
    else
    {
        Unsupported("light type " + std::to_string(l->type_index) +
                    " (supported: Point, Spot, UniformInfinite, DiffuseArea)");
    }
    return out;
}

// Rendering whose job runs the GPU render and then fills the Film.
class GpuRendering : public Rendering
{
public:
    explicit GpuRendering(const Camera* camera)
        : Rendering(camera)
    {
    }

    bool IsDone() const override { return done.load(std::memory_order_acquire); }
    void LogProgress() const override
    {
        std::fprintf(stdout, "\rGPU rendering: %s", IsDone() ? "done\n" : "running");
        std::fflush(stdout);
    }

    Film& MutableFilm() { return film; }
    std::atomic<bool> done{ false };
};

} // namespace

namespace bulbit_gpu
{

// ---------------------------------------------------------------- GpuBVH

GpuBVH::GpuBVH(const BVH& bvh)
{
    const std::vector<Primitive*>& prims = bvh.*Get(BvhPrims{});
    const auto* nodes = bvh.*Get(BvhNodes{}); // BVH::LinearBVHNode, a private type
    prims_.assign(prims.begin(), prims.end());
    // Nodes reachable from the root (the flattened array is dense, in DFS order).
    int32_t count = 0;
    std::vector<int32_t> stack{ 0 };
    while (!stack.empty() && !prims_.empty())
    {
        int32_t i = stack.back();
        stack.pop_back();
        ++count;
        if (nodes[i].primitive_count == 0)
        {
            stack.push_back(i + 1);
            stack.push_back(nodes[i].child2_offset);
        }
    }
    std::vector<bbg_bvh_node> flat(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i)
    {
        bbg_bvh_node& o = flat[i];
        std::memset(&o, 0, sizeof(o));
        Put3(o.bmin, nodes[i].aabb.min);
        Put3(o.bmax, nodes[i].aabb.max);
        o.offset = nodes[i].primitives_offset;
        o.count = nodes[i].primitive_count;
        o.axis = nodes[i].primitive_count == 0 ? nodes[i].axis : 0;
    }
    // The BVH keeps its primitives in leaf order, which is this accel's
    // primitive order, so slot i holds primitive i.
    std::vector<int32_t> slots(prims_.size());
    for (size_t i = 0; i < slots.size(); ++i)
    {
        slots[i] = int32_t(i);
    }
    bbg_bvh tree{ count, flat.data(), int32_t(slots.size()), slots.data() };
    Upload(&tree);
}

GpuBVH::GpuBVH(const std::vector<Primitive*>& primitives, GpuTree tree, float split_budget)
    : prims_(primitives.begin(), primitives.end())
{
    Upload(nullptr, tree, split_budget);
}

GpuBVH::~GpuBVH()
{
    if (accel_)
    {
        bbg_accel_destroy(accel_);
    }
}

void GpuBVH::Upload(const bbg_bvh* tree, GpuTree kind, float split_budget)
{
    std::vector<float> positions, normals, tangents, uvs;
    std::vector<int32_t> tri_indices, prim_kind, prim_index;
    std::vector<bbg_sphere> spheres;
    std::unordered_map<const Mesh*, int32_t> mesh_base;
    for (size_t i = 0; i < prims_.size(); ++i)
    {
        const Primitive* p = prims_[i];
        index_[p] = int32_t(i);
        const Shape* shape = p->GetShape();
        if (auto* tri = dynamic_cast<const Triangle*>(shape))
        {
            const Mesh* mesh = tri->*Get(TriMesh{});
            auto it = mesh_base.find(mesh);
            if (it == mesh_base.end())
            {
                const auto& pos = mesh->*Get(MeshPositions{});
                const auto& nrm = mesh->*Get(MeshNormals{});
                const auto& tan = mesh->*Get(MeshTangents{});
                const auto& uv = mesh->*Get(MeshUVs{});
                if (nrm.size() != pos.size() || tan.size() != pos.size() || uv.size() != pos.size())
                {
                    Unsupported("meshes need normals, tangents and uvs per vertex");
                }
                it = mesh_base.emplace(mesh, int32_t(positions.size() / 3)).first;
                for (size_t v = 0; v < pos.size(); ++v)
                {
                    positions.insert(positions.end(), { pos[v].x, pos[v].y, pos[v].z });
                    normals.insert(normals.end(), { nrm[v].x, nrm[v].y, nrm[v].z });
                    tangents.insert(tangents.end(), { tan[v].x, tan[v].y, tan[v].z });
                    uvs.insert(uvs.end(), { uv[v].x, uv[v].y });
                }
            }
            const int32* v = tri->*Get(TriV{});
            prim_kind.push_back(BBG_PRIM_TRIANGLE);
            prim_index.push_back(int32_t(tri_indices.size() / 3));
            for (int k = 0; k < 3; ++k)
            {
                tri_indices.push_back(it->second + v[k]);
            }
        }
        else if (auto* sph = dynamic_cast<const Sphere*>(shape))
        {
            bbg_sphere s{};
            Put3(s.p, sph->transform.p);
            s.q[0] = sph->transform.q.x;
            s.q[1] = sph->transform.q.y;
            s.q[2] = sph->transform.q.z;
            s.q[3] = sph->transform.q.w;
            Put3(s.s, sph->transform.s);
            s.radius = sph->radius;
            prim_kind.push_back(BBG_PRIM_SPHERE);
            prim_index.push_back(int32_t(spheres.size()));
            spheres.push_back(s);
        }
        else
        {
            Unsupported("shape type (supported: Triangle, Sphere)");
        }
        if (const Material* m = p->GetMaterial())
        {
            if (!OpaqueAlpha(m->GetAlphaTexture()))
            {
                Unsupported("materials with alpha below 1 (cut-outs)");
            }
        }
    }
    bbg_geometry g{};
    g.n_vertices = int32_t(positions.size() / 3);
    g.positions = positions.data();
    g.normals = normals.data();
    g.tangents = tangents.data();
    g.uvs = uvs.data();
    g.n_triangles = int32_t(tri_indices.size() / 3);
    g.tri_indices = tri_indices.data();
    g.n_spheres = int32_t(spheres.size());
    g.spheres = spheres.data();
    g.n_prims = int32_t(prims_.size());
    g.prim_kind = prim_kind.data();
    g.prim_index = prim_index.data();
    if (tree || kind == GpuTree::Reference || prims_.empty())
    {
        Check(bbg_accel_create(&g, tree, &accel_), "bbg_accel_create");
    }
    else if (kind == GpuTree::DeviceLinear)
    {
        Check(bbg_accel_create_device_build(&g, &accel_), "bbg_accel_create_device_build");
    }
    else if (kind == GpuTree::DeviceSah)
    {
        Check(bbg_accel_create_device_sah(&g, &accel_), "bbg_accel_create_device_sah");
    }
    else if (kind == GpuTree::DeviceSplitReferences)
    {
        Check(bbg_accel_create_device_split(&g, split_budget, &accel_), "bbg_accel_create_device_split");
    }
    else
    {
        Check(bbg_accel_create_split(&g, split_budget, &accel_), "bbg_accel_create_split");
    }
    float b[6];
    Check(bbg_accel_bounds(accel_, b), "bbg_accel_bounds");
    bounds_ = AABB(Point3(b[0], b[1], b[2]), Point3(b[3], b[4], b[5]));
}

AABB GpuBVH::GetAABB() const
{
    return bounds_;
}

int32_t GpuBVH::IndexOf(const Primitive* p) const
{
    auto it = index_.find(p);
    return it == index_.end() ? -1 : it->second;
}

namespace
{
bbg_ray ToRay(const Ray& ray, Float t_min, Float t_max)
{
    bbg_ray r{};
    Put3(r.o, ray.o);
    Put3(r.d, ray.d);
    r.t_min = t_min;
    r.t_max = t_max;
    return r;
}
} // namespace

bool GpuBVH::Intersect(Intersection* out_isect, const Ray& ray, Float t_min, Float t_max) const
{
    bbg_ray r = ToRay(ray, t_min, t_max);
    bbg_hit h{};
    {
        std::lock_guard<std::mutex> lock(mutex_);
        Check(bbg_intersect(accel_, &r, 1, &h, BBG_MEM_HOST, nullptr), "bbg_intersect");
    }
    if (h.prim < 0)
    {
        return false;
    }
    return prims_[h.prim]->Intersect(out_isect, ray, t_min, t_max);
}

bool GpuBVH::IntersectAny(const Ray& ray, Float t_min, Float t_max) const
{
    bbg_ray r = ToRay(ray, t_min, t_max);
    uint8_t occluded = 0;
    std::lock_guard<std::mutex> lock(mutex_);
    Check(bbg_intersect_any(accel_, &r, 1, &occluded, BBG_MEM_HOST, nullptr), "bbg_intersect_any");
    return occluded != 0;
}

void GpuBVH::IntersectBatch(const bbg_ray* rays, int64_t n, bbg_hit* hits) const
{
    std::lock_guard<std::mutex> lock(mutex_);
    Check(bbg_intersect(accel_, rays, n, hits, BBG_MEM_HOST, nullptr), "bbg_intersect");
}

void GpuBVH::OccludedBatch(const bbg_ray* rays, int64_t n, uint8_t* occluded) const
{
    std::lock_guard<std::mutex> lock(mutex_);
    Check(bbg_intersect_any(accel_, rays, n, occluded, BBG_MEM_HOST, nullptr), "bbg_intersect_any");
}

void GpuBVH::QueryBatches(const bbg_ray* rays, int64_t n, bbg_hit* hits, const bbg_ray* shadow_rays, int64_t m,
                          uint8_t* occluded) const
{
    std::lock_guard<std::mutex> lock(mutex_);
    bbg_status s = bbg_intersect_submit(accel_, rays, n, hits, BBG_MEM_HOST);
    if (s == BBG_OK)
    {
        s = bbg_intersect_any_submit(accel_, shadow_rays, m, occluded, BBG_MEM_HOST);
    }
    bbg_status w = bbg_accel_synchronize(accel_); // also after a failed submission: nothing stays queued
    Check(s != BBG_OK ? s : w, "bbg_intersect_submit");
}

// ---------------------------------------------------------------- GpuPathIntegrator

GpuPathIntegrator::GpuPathIntegrator(const GpuBVH* accel, std::vector<Light*> lights, const Sampler* sampler,
                                     int32 max_bounces, int32 rr_min_bounces, bool regularize_bsdf)
    : Integrator(accel, std::move(lights), std::make_unique<PowerLightSampler>())
    , gpu_{ accel }
    , sampler_{ sampler }
{
    if (!dynamic_cast<const IndependentSampler*>(sampler) && !dynamic_cast<const StratifiedSampler*>(sampler))
    {
        Unsupported("sampler (supported: IndependentSampler, StratifiedSampler)");
    }
    // Materials, deduplicated, and each primitive's index among them.
    std::vector<bbg_material> materials;
    std::unordered_map<const Material*, int32_t> mat_index;
    std::vector<int32_t> prim_material;
    for (const Primitive* p : accel->Primitives())
    {
        const Material* m = p->GetMaterial();
        if (!m)
        {
            prim_material.push_back(-1);
            continue;
        }
        auto it = mat_index.find(m);
        if (it == mat_index.end())
        {
            it = mat_index.emplace(m, int32_t(materials.size())).first;
            materials.push_back(TranslateMaterial(m));
        }
        prim_material.push_back(it->second);
    }
    std::vector<bbg_light> ls;
    for (const Light* l : all_lights)
    {
        ls.push_back(TranslateLight(l, *accel));
    }
    Check(bbg_integrator_create(accel->Handle(), prim_material.data(), materials.data(), int32_t(materials.size()),
                                ls.data(), int32_t(ls.size()), max_bounces, rr_min_bounces, regularize_bsdf ? 1 : 0,
                                &integrator_),
          "bbg_integrator_create");
}

GpuPathIntegrator::~GpuPathIntegrator()
{
    if (integrator_)
    {
        bbg_integrator_destroy(integrator_);
    }
}

Rendering* GpuPathIntegrator::Render(Allocator& alloc, const Camera* camera)
{
    auto* pc = dynamic_cast<const PerspectiveCamera*>(camera);
    const Filter* filter = pc ? pc->GetFilter() : nullptr;
    int32_t filter_type = -1;
    float filter_sigma = 0;
    if (dynamic_cast<const BoxFilter*>(filter))
    {
        filter_type = BBG_FILTER_BOX;
    }
    else if (dynamic_cast<const TentFilter*>(filter))
    {
        filter_type = BBG_FILTER_TENT;
    }
    else if (auto* gf = dynamic_cast<const GaussianFilter*>(filter))
    {
        filter_type = BBG_FILTER_GAUSSIAN;
        filter_sigma = gf->sigma;
    }
    if (!pc || filter_type < 0)
    {
        Unsupported("camera (supported: PerspectiveCamera with a Box, Tent or Gaussian filter)");
    }
    bbg_camera cam{};
    const Point2i res = pc->GetScreenResolution();
    cam.width = res.x;
    cam.height = res.y;
    Put3(cam.origin, pc->*Get(CamOrigin{}));
    Put3(cam.lower_left, pc->*Get(CamLowerLeft{}));
    Put3(cam.horizontal, pc->*Get(CamHorizontal{}));
    Put3(cam.vertical, pc->*Get(CamVertical{}));
    Put3(cam.u, pc->*Get(CamU{}));
    Put3(cam.v, pc->*Get(CamV{}));
    cam.lens_radius = pc->*Get(CamLensRadius{});
    cam.filter_extent = filter->extent;
    cam.filter_type = filter_type;
    cam.filter_sigma = filter_sigma;

    bbg_render_params params{};
    params.spp = sampler_->samples_per_pixel;
    params.use_graph = 1;
    if (auto* st = dynamic_cast<const StratifiedSampler*>(sampler_))
    {
        params.sampler = BBG_SAMPLER_STRATIFIED;
        params.seed = st->*Get(StratSeed{});
        params.x_samples = st->*Get(StratX{});
        params.jitter = (st->*Get(StratJitter{})) ? 1 : 0;
    }
    else
    {
        params.seed = static_cast<const IndependentSampler*>(sampler_)->*Get(SamplerSeed{});
    }

    GpuRendering* progress = alloc.new_object<GpuRendering>(camera);
    bbg_integrator* handle = integrator_;
    bbg_render_stats* stats = &stats_;
    progress->Start(RunAsync([=]() -> bool {
      try
      {
        const int64_t pixels = int64_t(cam.width) * cam.height;
        std::vector<float> rgb(3 * static_cast<size_t>(pixels)), moments(2 * static_cast<size_t>(pixels));
        std::vector<int32_t> count(static_cast<size_t>(pixels));
        bbg_film film{ rgb.data(), count.data(), moments.data(), nullptr };
        Check(bbg_render(handle, &cam, &params, &film, BBG_MEM_HOST, stats), "bbg_render");
        // The device film is Film::AddSample (src/reconstruction/film.cpp:26-38)
        // applied to every non-nullish sample of a pixel in sample order, as
        // UniDirectionalRayIntegrator::Render calls it (src/integrator/integrator.cpp:183-197),
        // starting from the zeroed film the constructor leaves: its sums, counts
        // and luminance moments are the Film's state, stored as they are.
        Film& f = progress->MutableFilm();
        Spectrum* samples = (f.*Get(FilmSamples{})).get();
        int32* counts = (f.*Get(FilmCounts{})).get();
        Point2* mom = (f.*Get(FilmMoments{})).get();
        ParallelFor(0, cam.height, [&](int32 y) {
            for (int64_t p = int64_t(y) * cam.width; p < int64_t(y + 1) * cam.width; ++p)
            {
                samples[p] = Spectrum(rgb[3 * p], rgb[3 * p + 1], rgb[3 * p + 2]);
                counts[p] = count[p];
                mom[p] = Point2(moments[2 * p], moments[2 * p + 1]);
            }
        });
        progress->done.store(true, std::memory_order_release);
        return true;
      }
      catch (const std::exception& e)
      {
        // The job runs on the reference's thread pool: report, finish, and
        // leave the film empty rather than end the process.
        std::fprintf(stderr, "%s\n", e.what());
        progress->done.store(true, std::memory_order_release);
        return false;
      }
    }));
    return progress;
}

Integrator* CreateGpuIntegrator(Allocator& alloc, const IntegratorInfo& info, const GpuBVH* accel,
                                const std::vector<Light*>& lights, const Sampler* sampler)
{
    if (info.type != IntegratorType::path)
    {
        return nullptr;
    }
    return alloc.new_object<GpuPathIntegrator>(accel, lights, sampler, info.max_bounces, info.rr_min_bounces,
                                               info.regularize_bsdf);
}

} // namespace bulbit_gpu
