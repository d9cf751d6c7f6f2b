// Internal layouts shared by the host code and the CUDA kernels of
// bulbit-b200. Nothing here crosses the C ABI (include/bbg.h does).
#pragma once

#include "bbg.h"

#include <cstdint>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define BBG_HD __host__ __device__ __forceinline__
#else
#define BBG_HD inline
#endif

namespace bbg
{

// Traversal stack capacity per ray. The reference's stack grows on the heap
// past 64 entries (include/bulbit/bvh.h:107); here a tree whose depth needs
// more is rejected at upload (BBG_ERR_STACK_OVERFLOW) so no kernel can
// overflow.
constexpr int kStackCapacity = 64;

// Slot record: 48 bytes per leaf slot, the primitive's intersection data
// copied into leaf order so one leaf test is three 16-byte loads.
//   triangle: (p0.xyz, prim) (p1.xyz, 0) (p2.xyz, 0)
//   sphere:   (p.xyz, prim | kSphereBit) (q.xyzw) (s.xyz, radius)
constexpr uint32_t kSphereBit = 0x80000000u;

// Per-primitive shading record.
struct PrimInfo
{
    int32_t kind;       // BBG_PRIM_*
    int32_t index;      // triangle or sphere number
    int32_t material;   // material index or -1
    int32_t area_light; // light index of the DiffuseAreaLight on it, or -1
};

// Device material: the BxDF the reference material builds, with its
// constructor-time derived values (include/bulbit/bxdfs.h).
struct MaterialDev
{
    int32_t type;     // BBG_MAT_*
    int32_t flags;    // BxDF_Flags of the BxDF (include/bulbit/bxdf.h:8)
    float r[3];       // Lambertian r / conductor reflectance / dielectric Sqrt(r) / MR color
    float eta[3];     // conductor eta; dielectric eta in eta[0]
    float k[3];       // conductor k
    float alpha_x;    // microfacet alpha (after RoughnessToAlpha)
    float alpha_y;
    float metallic;
    int32_t ms;       // conductor: energy compensation (ConductorMultiScatteringBxDF)
};

// BxDF_Flags values (include/bulbit/bxdf.h:8-22).
enum : int32_t
{
    kFlagReflection = 1,
    kFlagTransmission = 2,
    kFlagDiffuse = 4,
    kFlagGlossy = 8,
    kFlagSpecular = 16
};

// Device light: constructor and Preprocess results of the reference lights.
struct LightDev
{
    int32_t type;      // BBG_LIGHT_*
    int32_t prim;      // area light primitive
    int32_t two_sided;
    int32_t pad;
    float p[3];        // point/spot position
    float frame_x[3];  // spot light frame (Frame(-Normalize(direction)))
    float frame_y[3];
    float frame_z[3];
    float cos_theta_min, cos_theta_max;
    float L[3];        // point/spot intensity; infinite l; area emission
    float scale;       // infinite light scale
    float world_center[3];
    float world_radius;
};

struct CameraDev
{
    int32_t width, height;
    float origin[3], lower_left[3], horizontal[3], vertical[3], u[3], v[3];
    float lens_radius;
    float filter_extent;
    int32_t filter_type;     // BBG_FILTER_*
    const float* filter_cdf; // Gaussian: GaussianFilterCdf tables (device)
};

// Gaussian filter table resolution (GaussianFilter: 32 x 32 samples).
constexpr int32_t kFilterTable = 32;
constexpr int32_t kFilterCdfFloats = (kFilterTable + 1) * (kFilterTable + 1);
void GaussianFilterCdf(float sigma, float extent, float* cdf_out);

// ---- host helpers (host_build.cpp) -----------------------------------------

void SetError(const char* fmt, ...);
bbg_status Fail(bbg_status s, const char* fmt, ...);

// Reference-exact host computations.
void PrimAabbs(const bbg_geometry& g, float* aabbs);
bbg_status BuildBvh(const float* aabbs, int32_t n, bbg_bvh_node* nodes, int32_t* slots, int32_t* n_nodes);
// Index and pointer checks of a geometry record (counts, vertex and
// primitive references in range).
bbg_status CheckGeometry(const bbg_geometry* g);
// Reference splitting before the SAH build (see host_build.cpp): references
// (box, primitive) for every primitive, with poorly filled triangle boxes
// split up to `budget` extra references per primitive.
bbg_status SplitReferences(const bbg_geometry& g, float budget, std::vector<float>* ref_aabbs,
                           std::vector<int32_t>* ref_prims);
bbg_status ValidateBvh(const bbg_bvh_node* nodes, int32_t n_nodes, int32_t n_slots, int32_t n_prims,
                       const int32_t* slot_prims, int32_t* max_depth);
void CameraFromSpec(const bbg_camera_spec& s, bbg_camera* out);
bbg_status MakeMaterial(const bbg_material& m, MaterialDev* out);
// Light constructor + Preprocess(world bounds) + power (Phi luminance).
bbg_status MakeLight(const bbg_light& l, const bbg_geometry& g, const float world_aabb[6], LightDev* out,
                     float* power_luminance);
// Distribution1D (include/bulbit/sampling.h:343-424) over the light powers:
// func (n), cdf (n+1), func_integral.
void BuildDistribution(const float* f, int32_t n, float* func, float* cdf, float* func_integral);
// Walker alias table with the same pmf: prob (n), alias (n).
void BuildAlias(const float* pmf, int32_t n, float* prob, int32_t* alias);

} // namespace bbg
