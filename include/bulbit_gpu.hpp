// C++ drop-in for the reference renderer's ray-query and path-tracing path
// (Sopiro/Bulbit), on top of the C ABI in bbg.h.
//
// A program written against the reference library changes two lines:
//
//     BVH accel(scene.GetPrimitives());                       // unchanged
//     bulbit_gpu::GpuBVH gpu_accel(accel);                     // + GPU copy of that tree
//     bulbit_gpu::GpuPathIntegrator integrator(&gpu_accel, scene.GetLights(), &sampler, max_bounces);
//     Rendering* rendering = integrator.Render(alloc, &camera); // same call, same Rendering/Film
//
// GpuBVH is an Intersectable beside BVH (include/bulbit/bvh.h:11-75): it
// takes the reference-built SAH tree node for node (or builds the same tree
// itself from the primitives) and answers Intersect / IntersectAny
// (include/bulbit/intersectable.h:37-45) on the GPU, one ray at a time
// through the batched kernel, or in batches through IntersectBatch /
// OccludedBatch. GpuPathIntegrator is an Integrator with PathIntegrator's
// constructor (include/bulbit/integrators.h:92-114): the base constructor
// preprocesses the lights exactly as the reference does, and Render()
// returns at once a Rendering whose job renders on the GPU and leaves its Film
// in the state Film::AddSample leaves after the reference's samples in the
// reference's order (sums, counts and luminance moments, accumulated on the
// device per pixel in sample order), the state the reference's Render() would
// leave, up to the per-path tolerance of the GPU arithmetic.
//
// Supported scene content (checked in the constructors, which throw
// std::runtime_error otherwise): Triangle and Sphere shapes; DiffuseMaterial,
// ConductorMaterial and DielectricMaterial (energy compensation on or off)
// and MetallicRoughnessMaterial with constant textures and no normal maps
// (alpha only as a constant not below 1, which the alpha test never cuts;
// DiffuseMaterial roughness only as a constant not above 0, Lambertian);
// PointLight, SpotLight, UniformInfiniteLight, DiffuseAreaLight with a
// constant emission; PerspectiveCamera with a Box, Tent or Gaussian filter;
// IndependentSampler or StratifiedSampler.
// Primitives without a material are passed through as the reference does.
//
// Build: compile bulbit_b200/cpp/bulbit_gpu.cpp with the reference's include
// directory and flags, link libbulbit_b200.so and the reference library.
#pragma once

#include "bbg.h"

#include "bulbit/bulbit.h"
#include "bulbit/bvh.h"
#include "bulbit/cameras.h"
#include "bulbit/integrator.h"
#include "bulbit/lights.h"
#include "bulbit/materials.h"
#include "bulbit/progress.h"
#include "bulbit/renderer_info.h"
#include "bulbit/samplers.h"
#include "bulbit/shapes.h"

#include <atomic>
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace bulbit_gpu
{

// The tree a GpuBVH built from a primitive list uses. Reference: the same
// SAH tree as BVH::BVH (hits identical to the reference's), built on the
// host. DeviceSah: that same tree, node for node, built on the GPU in
// milliseconds. DeviceLinear: a linear BVH built on the GPU. SplitReferences:
// the SAH build over split triangle references (faster traversal of long or
// diagonal triangles, a host build of seconds). DeviceSplitReferences: split
// references and the SAH build over them, both on the GPU (a fraction of a
// second on millions of triangles). The last three change only which of two
// hits at exactly the same t is returned.
enum class GpuTree
{
    Reference,
    DeviceLinear,
    SplitReferences,
    DeviceSah,
    DeviceSplitReferences
};

class GpuBVH : public bulbit::Intersectable
{
public:
    // The reference's own tree (BVH::nodes, BVH::primitives), node for node.
    explicit GpuBVH(const bulbit::BVH& bvh);
    // A tree built by the library from the primitives, in the order given
    // (primitive index = position): by default the same SAH tree as
    // BVH::BVH (bbg_bvh_build); split_budget = extra references per
    // primitive for GpuTree::SplitReferences and DeviceSplitReferences.
    explicit GpuBVH(const std::vector<bulbit::Primitive*>& primitives, GpuTree tree = GpuTree::Reference,
                    float split_budget = 3.0f);
    ~GpuBVH() override;

    GpuBVH(const GpuBVH&) = delete;
    GpuBVH& operator=(const GpuBVH&) = delete;

    bulbit::AABB GetAABB() const override;
    // One ray through the GPU kernel; the hit's record (point, normals, uv,
    // front face) is completed by the hit primitive's own Intersect, so it is
    // the record the reference's BVH::Intersect returns for that primitive.
    bool Intersect(bulbit::Intersection* out_isect, const bulbit::Ray& ray, ::Float t_min,
                   ::Float t_max) const override;
    bool IntersectAny(const bulbit::Ray& ray, ::Float t_min, ::Float t_max) const override;

    // Batched queries, host buffers: closest hits (hit.prim indexes
    // Primitives(), -1 on a miss) and occlusion flags. All queries of one
    // GpuBVH are serialised (the reference calls Intersect from every pool
    // thread; one call at a time uses the accel's staging buffers).
    void IntersectBatch(const bbg_ray* rays, int64_t n, bbg_hit* hits) const;
    void OccludedBatch(const bbg_ray* rays, int64_t n, uint8_t* occluded) const;
    // Both batches submitted at once, then waited for: the shadow rays'
    // upload overlaps the closest-hit traversal (bbg_intersect_submit,
    // bbg_intersect_any_submit, bbg_accel_synchronize). Results equal
    // IntersectBatch's and OccludedBatch's; from page-locked buffers the
    // copies run while the other batch is traced.
    void QueryBatches(const bbg_ray* rays, int64_t n, bbg_hit* hits, const bbg_ray* shadow_rays, int64_t m,
                      uint8_t* occluded) const;

    const std::vector<const bulbit::Primitive*>& Primitives() const { return prims_; }
    int32_t IndexOf(const bulbit::Primitive* p) const;
    bbg_accel* Handle() const { return accel_; }

private:
    void Upload(const bbg_bvh* tree, GpuTree kind = GpuTree::Reference, float split_budget = 0.0f);

    std::vector<const bulbit::Primitive*> prims_;
    std::unordered_map<const bulbit::Primitive*, int32_t> index_;
    bbg_accel* accel_ = nullptr;
    bulbit::AABB bounds_;
    mutable std::mutex mutex_;
};

class GpuPathIntegrator : public bulbit::Integrator
{
public:
    // PathIntegrator(accel, lights, sampler, max_bounces, rr_min_bounces,
    // regularize_bsdf) with the GPU accel in place of the BVH.
    GpuPathIntegrator(const GpuBVH* accel, std::vector<bulbit::Light*> lights, const bulbit::Sampler* sampler,
                      ::int32 max_bounces, ::int32 rr_min_bounces = 1, bool regularize_bsdf = false);
    ~GpuPathIntegrator() override;

    // Returns at once; the Rendering's job renders on the GPU. Wait() /
    // WaitAndLogProgress() and GetFilm() behave as for the reference.
    bulbit::Rendering* Render(::Allocator& alloc, const bulbit::Camera* camera) override;

    // Device time and ray counts of the last finished render.
    const bbg_render_stats& LastStats() const { return stats_; }
    bbg_integrator* Handle() const { return integrator_; }

private:
    const GpuBVH* gpu_;
    const bulbit::Sampler* sampler_;
    bbg_integrator* integrator_ = nullptr;
    bbg_render_stats stats_{};
};

// Integrator::Create (src/integrator/integrator.cpp:16-31) with the GPU
// accel: IntegratorType::path gives a GpuPathIntegrator with the info's
// max_bounces, rr_min_bounces and regularize_bsdf, allocated from alloc
// (released with alloc.delete_object, as the reference's callers do). The
// other integrator types have no GPU implementation here: nullptr, which is
// what Integrator::Create returns for a type it cannot make.
bulbit::Integrator* CreateGpuIntegrator(::Allocator& alloc, const bulbit::IntegratorInfo& info, const GpuBVH* accel,
                                        const std::vector<bulbit::Light*>& lights, const bulbit::Sampler* sampler);

} // namespace bulbit_gpu
