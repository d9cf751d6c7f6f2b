// Drop-in check of include/bulbit_gpu.hpp: scenes built with the reference's
// own Scene API, as a library user would, then queried and rendered through
// the reference classes (BVH, PathIntegrator) and through the GPU drop-ins
// (GpuBVH, GpuPathIntegrator). Prints one JSON line with the comparison and
// exits non-zero when a check fails. Run by tests/test_dropin_gpu.py; built by
// oracle/Makefile (it links the reference library, so it is test-only).
//
// Checks:
//  * GpuBVH::Intersect returns the same primitive and record (t, point,
//    normals, uv, front face) as BVH::Intersect, and IntersectAny the same
//    answer, on random rays; IntersectBatch agrees with both;
//  * GpuPathIntegrator::Render leaves a Film whose sample counts equal the
//    reference's and whose pixel sums agree within 1e-3 relative for 99.5 %
//    of pixels (per-path tolerance 1e-4 of the GPU arithmetic, summed), with
//    equal image means within 1e-3 relative.

#include "bulbit_gpu.hpp"

#include "bulbit/parallel_for.h"
#include "bulbit/random.h"

#include <cmath>
#include <cstdio>
#include <string>

using namespace bulbit;

namespace
{

struct Result
{
    bool ok = true;
    std::string json;
    void Add(const std::string& key, double v)
    {
        char buf[128];
        std::snprintf(buf, sizeof(buf), "%s\"%s\": %.9g", json.empty() ? "" : ", ", key.c_str(), v);
        json += buf;
    }
    void Expect(bool cond, const std::string& key)
    {
        Add(key, cond ? 1 : 0);
        ok = ok && cond;
    }
};

// The README scene: a red sphere under a spot light and a uniform sky.
void ReadmeScene(Scene& scene)
{
    Texture<Spectrum>* tex = scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(0.85f, 0.2f, 0.2f));
    Material* mat = scene.CreateMaterial<DiffuseMaterial>(tex);
    Point3 sphere_pos(0.0f, 1.0f, 0.0f);
    scene.CreatePrimitive(scene.CreateShape<Sphere>(sphere_pos, 1.0f), mat, MediumInterface{});
    Point3 light_pos(2.5f, 4.0f, 2.0f);
    scene.CreateLight<SpotLight>(light_pos, Normalize(light_pos - sphere_pos), Spectrum(80.0f), 35.0f, 20.0f,
                                 nullptr);
    scene.CreateLight<UniformInfiniteLight>(Spectrum(0.1f));
}

// A box of two meshes (floor + walls, and a block of random triangles)
// with a conductor, a dielectric and a ceiling area light.
void MeshScene(Scene& scene)
{
    auto quad_mesh = [&](std::vector<Point3> pts) {
        std::vector<Vec3> n, t;
        std::vector<Point2> uv;
        std::vector<int32> idx;
        for (size_t q = 0; q < pts.size(); q += 4)
        {
            Vec3 nn = Normalize(Cross(pts[q + 1] - pts[q], pts[q + 2] - pts[q]));
            Vec3 tt = Normalize(pts[q + 1] - pts[q]);
            for (int k = 0; k < 4; ++k)
            {
                n.push_back(nn);
                t.push_back(tt);
                uv.push_back(Point2(0, 0));
            }
            int32 b = int32(q);
            idx.insert(idx.end(), { b, b + 1, b + 2, b, b + 2, b + 3 });
        }
        return scene.CreateMesh(std::move(pts), std::move(n), std::move(t), std::move(uv), std::move(idx),
                                Mat4(identity));
    };
    // Floor, back wall, ceiling (inward facing) and a small light quad.
    Mesh* box = quad_mesh({ Point3(-2, 0, -2), Point3(-2, 0, 2), Point3(2, 0, 2), Point3(2, 0, -2),
                            Point3(-2, 0, -2), Point3(2, 0, -2), Point3(2, 3, -2), Point3(-2, 3, -2),
                            Point3(-2, 3, -2), Point3(2, 3, -2), Point3(2, 3, 2), Point3(-2, 3, 2),
                            Point3(-0.5f, 2.99f, -0.5f), Point3(0.5f, 2.99f, -0.5f), Point3(0.5f, 2.99f, 0.5f),
                            Point3(-0.5f, 2.99f, 0.5f) });
    auto* white = scene.CreateMaterial<DiffuseMaterial>(
        scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(0.7f, 0.7f, 0.65f)));
    // Gold with the library default (energy_compensation = true).
    auto* gold = scene.CreateMaterial<ConductorMaterial>(
        scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(0.161f, 0.492f, 1.426f)),
        scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(4.08769f, 2.32625f, 1.846f)),
        scene.CreateTexture<ConstantTexture, Float>(0.3f), scene.CreateTexture<ConstantTexture, Float>(0.3f));
    // Rough glass, also with the library default (energy_compensation = true).
    auto* glass = scene.CreateMaterial<DielectricMaterial>(
        1.5f, scene.CreateTexture<ConstantTexture, Float>(0.25f), scene.CreateTexture<ConstantTexture, Float>(0.25f),
        scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(1.0f)));
    std::vector<Primitive*> light_prims;
    for (int32 i = 0; i < 8; ++i)
    {
        Primitive* p = scene.CreatePrimitive(scene.CreateShape<Triangle>(box, size_t(i)), white, MediumInterface{});
        if (i >= 6)
        {
            light_prims.push_back(p);
        }
    }
    // A block of random triangles (second mesh).
    RNG rng(7);
    std::vector<Point3> pts;
    for (int32 i = 0; i < 300; ++i)
    {
        Point3 c(rng.NextFloat() * 2 - 1, rng.NextFloat() * 1.5f + 0.2f, rng.NextFloat() * 2 - 1);
        for (int k = 0; k < 3; ++k)
        {
            pts.push_back(c + Vec3(rng.NextFloat() - 0.5f, rng.NextFloat() - 0.5f, rng.NextFloat() - 0.5f) * 0.3f);
        }
    }
    std::vector<Vec3> n, t;
    std::vector<Point2> uv;
    std::vector<int32> idx;
    for (size_t i = 0; i < pts.size(); i += 3)
    {
        Vec3 nn = Normalize(Cross(pts[i + 1] - pts[i], pts[i + 2] - pts[i]));
        Vec3 tt = Normalize(pts[i + 1] - pts[i]);
        for (int k = 0; k < 3; ++k)
        {
            n.push_back(nn);
            t.push_back(tt);
            uv.push_back(Point2(0.25f * k, 0.5f));
            idx.push_back(int32(i) + k);
        }
    }
    Mesh* block = scene.CreateMesh(std::move(pts), std::move(n), std::move(t), std::move(uv), std::move(idx),
                                   Mat4(identity));
    for (int32 i = 0; i < 300; ++i)
    {
        const Material* m = i % 2 ? static_cast<const Material*>(gold) : static_cast<const Material*>(glass);
        scene.CreatePrimitive(scene.CreateShape<Triangle>(block, size_t(i)), m, MediumInterface{});
    }
    scene.CreatePrimitive(scene.CreateShape<Sphere>(Point3(1.2f, 0.5f, 0.8f), 0.5f), gold, MediumInterface{});
    for (Primitive* p : light_prims)
    {
        scene.CreateLight<DiffuseAreaLight>(
            p, scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(17.0f, 12.0f, 4.0f)), false);
    }
}

void CompareQueries(const BVH& bvh, const bulbit_gpu::GpuBVH& gpu, Point3 center, Float radius, Result* r,
                    const std::string& tag)
{
    RNG rng(11);
    const int n_single = 2000, n_batch = 100000;
    std::vector<Ray> rays;
    for (int i = 0; i < n_batch; ++i)
    {
        Vec3 a(rng.NextFloat() * 2 - 1, rng.NextFloat() * 2 - 1, rng.NextFloat() * 2 - 1);
        Vec3 b(rng.NextFloat() * 2 - 1, rng.NextFloat() * 2 - 1, rng.NextFloat() * 2 - 1);
        Point3 o = center + a * radius;
        Point3 target = center + b * (radius * 0.4f);
        rays.push_back(Ray(o, Normalize(target - o)));
    }
    int same_single = 0, same_any = 0;
    for (int i = 0; i < n_single; ++i)
    {
        Intersection a{}, b{};
        bool ha = bvh.Intersect(&a, rays[i], Ray::epsilon, infinity);
        bool hb = gpu.Intersect(&b, rays[i], Ray::epsilon, infinity);
        bool same = ha == hb;
        if (same && ha)
        {
            same = a.primitive == b.primitive && a.t == b.t && a.point == b.point && a.normal == b.normal &&
                   a.uv == b.uv && a.front_face == b.front_face && a.shading.normal == b.shading.normal &&
                   a.shading.tangent == b.shading.tangent;
        }
        same_single += same;
        Float tmax = ha ? a.t * 0.5f : 10.0f;
        same_any += bvh.IntersectAny(rays[i], Ray::epsilon, tmax) == gpu.IntersectAny(rays[i], Ray::epsilon, tmax);
    }
    std::vector<bbg_ray> br(n_batch);
    for (int i = 0; i < n_batch; ++i)
    {
        br[i] = bbg_ray{ { rays[i].o.x, rays[i].o.y, rays[i].o.z },
                         { rays[i].d.x, rays[i].d.y, rays[i].d.z },
                         Ray::epsilon,
                         infinity };
    }
    std::vector<bbg_hit> hits(n_batch);
    gpu.IntersectBatch(br.data(), n_batch, hits.data());
    std::atomic<int> same_batch{ 0 };
    ParallelFor(0, n_batch, [&](int32 i) {
        Intersection a{};
        bool ha = bvh.Intersect(&a, rays[i], Ray::epsilon, infinity);
        bool same = ha == (hits[i].prim >= 0) && (!ha || (gpu.Primitives()[hits[i].prim] == a.primitive &&
                                                          hits[i].t == a.t));
        same_batch += same;
    });
    // Both batches submitted together give the separate calls' results.
    std::vector<bbg_ray> shadow(br);
    for (int i = 0; i < n_batch; ++i)
    {
        shadow[i].t_max = hits[i].prim >= 0 ? hits[i].t * 0.5f : 10.0f;
    }
    std::vector<uint8_t> occ(n_batch), occ_pair(n_batch);
    std::vector<bbg_hit> hits_pair(n_batch);
    gpu.OccludedBatch(shadow.data(), n_batch, occ.data());
    gpu.QueryBatches(br.data(), n_batch, hits_pair.data(), shadow.data(), n_batch, occ_pair.data());
    bool pair_same = occ == occ_pair;
    for (int i = 0; i < n_batch && pair_same; ++i)
    {
        pair_same = hits_pair[i].prim == hits[i].prim && hits_pair[i].t == hits[i].t && hits_pair[i].u == hits[i].u &&
                    hits_pair[i].v == hits[i].v;
    }
    r->Add(tag + "_single_same", same_single / double(n_single));
    r->Add(tag + "_any_same", same_any / double(n_single));
    r->Add(tag + "_batch_same", same_batch / double(n_batch));
    r->Add(tag + "_paired_batches_same", pair_same ? 1.0 : 0.0);
    r->Expect(same_single >= n_single - 2 && same_any >= n_single - 2 && same_batch >= n_batch - 20 && pair_same,
              tag + "_queries_ok");
}

void CompareRender(Scene& scene, const BVH& bvh, const bulbit_gpu::GpuBVH& gpu, const Camera& camera,
                   const Sampler& sampler, int32 bounces, Result* r, const std::string& tag)
{
    Allocator alloc;
    PathIntegrator cpu(&bvh, scene.GetLights(), &sampler, bounces);
    Rendering* a = cpu.Render(alloc, &camera);
    a->Wait();
    bulbit_gpu::GpuPathIntegrator gpi(&gpu, scene.GetLights(), &sampler, bounces);
    Rendering* b = gpi.Render(alloc, &camera);
    b->Wait();
    Image3 ia = a->GetFilm().GetRenderedImage();
    Image3 ib = b->GetFilm().GetRenderedImage();
    const int32 w = camera.GetScreenResolution().x, h = camera.GetScreenResolution().y;
    double mean_a = 0, mean_b = 0;
    int close = 0;
    for (int32 y = 0; y < h; ++y)
    {
        for (int32 x = 0; x < w; ++x)
        {
            Spectrum pa = ia(x, y), pb = ib(x, y);
            mean_a += pa.Luminance();
            mean_b += pb.Luminance();
            double d = std::max({ std::fabs(pa.r - pb.r), std::fabs(pa.g - pb.g), std::fabs(pa.b - pb.b) });
            close += d <= 1e-3 * std::max(1.0, double(pa.MaxComponent()));
        }
    }
    mean_a /= double(w) * h;
    mean_b /= double(w) * h;
    r->Add(tag + "_mean_reference", mean_a);
    r->Add(tag + "_mean_gpu", mean_b);
    r->Add(tag + "_pixels_close", close / (double(w) * h));
    r->Add(tag + "_gpu_device_ms", gpi.LastStats().device_ms);
    r->Expect(std::fabs(mean_a - mean_b) <= 1e-3 * mean_a && close >= 0.995 * w * h, tag + "_render_ok");
    alloc.delete_object(a);
    alloc.delete_object(b);
}

// Which constant textures the drop-in accepts: a roughness of 0 (Lambertian,
// src/material/diffuse_material.cpp:22-33) and an alpha of 1 (never cut,
// include/bulbit/primitive.h:60-66) are accepted, as the reference CLI's
// material builders attach them; a roughness above 0 (EONBxDF) and an alpha
// below 1 (cut-outs) are refused with an exception.
void CheckMaterialAcceptance(Result* r)
{
    auto attempt = [](Float roughness, Float alpha) {
        Scene scene;
        auto* mat = scene.CreateMaterial<DiffuseMaterial>(
            scene.CreateTexture<ConstantTexture, Spectrum>(Spectrum(0.5f)),
            scene.CreateTexture<ConstantTexture, Float>(roughness), nullptr,
            scene.CreateTexture<ConstantTexture, Float>(alpha));
        scene.CreatePrimitive(scene.CreateShape<Sphere>(Point3(0, 0, 0), 1.0f), mat, MediumInterface{});
        scene.CreateLight<UniformInfiniteLight>(Spectrum(1.0f));
        IndependentSampler sampler(1);
        try
        {
            bulbit_gpu::GpuBVH gpu(scene.GetPrimitives());
            bulbit_gpu::GpuPathIntegrator integrator(&gpu, scene.GetLights(), &sampler, 2);
        }
        catch (const std::runtime_error&)
        {
            return false;
        }
        return true;
    };
    r->Expect(attempt(0.0f, 1.0f), "material_opaque_lambertian_accepted_ok");
    r->Expect(!attempt(0.3f, 1.0f), "material_eon_refused_ok");
    r->Expect(!attempt(0.0f, 0.5f), "material_cutout_refused_ok");
}

} // namespace

int main()
{
    ThreadPool::global_thread_pool = std::make_unique<ThreadPool>(std::thread::hardware_concurrency());
    Result r;
    try
    {
        {
            Scene scene;
            ReadmeScene(scene);
            BVH bvh(scene.GetPrimitives());
            bulbit_gpu::GpuBVH gpu(bvh);
            CompareQueries(bvh, gpu, Point3(0, 1, 0), 3.0f, &r, "readme");
            BoxFilter filter;
            Point3 camera_pos(3.0f, 2.0f, 5.0f), sphere_pos(0.0f, 1.0f, 0.0f);
            PerspectiveCamera camera(Transform::LookAt(camera_pos, sphere_pos, y_axis), 35, 0.01f,
                                     Dist(camera_pos, sphere_pos), Point2i(160, 90), nullptr, &filter);
            IndependentSampler sampler(16);
            CompareRender(scene, bvh, gpu, camera, sampler, 8, &r, "readme");
        }
        {
            Scene scene;
            MeshScene(scene);
            BVH bvh(scene.GetPrimitives());
            bulbit_gpu::GpuBVH gpu(bvh);
            bulbit_gpu::GpuBVH gpu_own(scene.GetPrimitives()); // the library's own build of the same tree
            // Other trees over the same primitives (hits equal except exact ties).
            bulbit_gpu::GpuBVH gpu_split(scene.GetPrimitives(), bulbit_gpu::GpuTree::SplitReferences, 2.0f);
            bulbit_gpu::GpuBVH gpu_dev(scene.GetPrimitives(), bulbit_gpu::GpuTree::DeviceLinear);
            // The reference's SAH tree built on the GPU: identical records to BVH.
            bulbit_gpu::GpuBVH gpu_dev_sah(scene.GetPrimitives(), bulbit_gpu::GpuTree::DeviceSah);
            // Split references and their SAH tree, both built on the GPU.
            bulbit_gpu::GpuBVH gpu_dev_split(scene.GetPrimitives(), bulbit_gpu::GpuTree::DeviceSplitReferences, 2.0f);
            CompareQueries(bvh, gpu, Point3(0, 1.2f, 0), 2.5f, &r, "mesh");
            CompareQueries(bvh, gpu_own, Point3(0, 1.2f, 0), 2.5f, &r, "mesh_own_tree");
            CompareQueries(bvh, gpu_split, Point3(0, 1.2f, 0), 2.5f, &r, "mesh_split_tree");
            CompareQueries(bvh, gpu_dev, Point3(0, 1.2f, 0), 2.5f, &r, "mesh_device_tree");
            CompareQueries(bvh, gpu_dev_sah, Point3(0, 1.2f, 0), 2.5f, &r, "mesh_device_sah_tree");
            CompareQueries(bvh, gpu_dev_split, Point3(0, 1.2f, 0), 2.5f, &r, "mesh_device_split_tree");
            // The camera's default filter (GaussianFilter) and a stratified sampler.
            GaussianFilter filter;
            Point3 eye(0.0f, 1.5f, 5.0f), at(0.0f, 1.2f, 0.0f);
            PerspectiveCamera camera(Transform::LookAt(eye, at, y_axis), 50, 0.0f, Dist(eye, at), Point2i(96, 72),
                                     nullptr, &filter);
            StratifiedSampler sampler(8, 4, true, 3);
            CompareRender(scene, bvh, gpu, camera, sampler, 12, &r, "mesh");
        }
        CheckMaterialAcceptance(&r);
    }
    catch (const std::exception& e)
    {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
    std::printf("{%s, \"ok\": %d}\n", r.json.c_str(), r.ok ? 1 : 0);
    return r.ok ? 0 : 1;
}
