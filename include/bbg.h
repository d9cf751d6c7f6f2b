/*
 * bbg.h — C ABI of bulbit-b200, a B200 (sm_100a) wavefront implementation of
 * Bulbit's unidirectional path tracer: SAH-BVH closest-hit / any-hit traversal
 * over triangles and spheres, and PathIntegrator's next-event estimation with
 * continuation-ray MIS.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, never
 * throws, and reports failure through a bbg_status code plus a thread-local
 * message (bbg_last_error). Handles own their device memory; callers own every
 * buffer they pass. Calls on one handle must not run concurrently.
 *
 * Reference interfaces each entry point replaces (paths inside Sopiro/Bulbit):
 *   bbg_bvh_build          BVH::BVH / BuildRecursive / FlattenBVH
 *                          (src/accel/bvh.cpp:8,56,273)
 *   bbg_accel_create       the GPU accel beside BVH: takes the reference-built
 *                          flattened tree (include/bulbit/bvh.h:46 layout) or
 *                          builds the same tree itself
 *   bbg_accel_create_device_sah  BVH::BVH (src/accel/bvh.cpp:8-297): the same
 *                          tree, node for node, built on the device
 *   bbg_intersect          BVH::Intersect (src/accel/bvh.cpp:299), batched
 *   bbg_intersect_any      BVH::IntersectAny (src/accel/bvh.cpp:334), batched
 *   bbg_accel_bounds       Intersectable::GetAABB (include/bulbit/intersectable.h:41)
 *   bbg_camera_perspective PerspectiveCamera::PerspectiveCamera
 *                          (src/camera/perspective_camera.cpp:8)
 *   bbg_integrator_create  PathIntegrator::PathIntegrator
 *                          (src/integrator/path_integrator.cpp:11) together with
 *                          Integrator::Integrator (src/integrator/integrator.cpp:107)
 *   bbg_render             UniDirectionalRayIntegrator::Render
 *                          (src/integrator/integrator.cpp:162) driving
 *                          PathIntegrator::Li (src/integrator/path_integrator.cpp:26),
 *                          filling the same per-pixel state as Film::AddSample
 *                          (src/reconstruction/film.cpp:26)
 *   bbg_sampler_draws      IndependentSampler::StartPixelSample / Next1D
 *                          (src/sampler/independent_sampler.cpp:13-22)
 */
#ifndef BBG_H
#define BBG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bbg_status
{
    BBG_OK = 0,
    BBG_ERR_INVALID_ARG = 1,    /* bad pointer, size or enum value */
    BBG_ERR_OOM = 2,            /* device allocation failed */
    BBG_ERR_TIMEOUT = 3,        /* a bounded device loop hit its iteration cap */
    BBG_ERR_QUEUE_OVERFLOW = 4, /* a wavefront queue exceeded its capacity */
    BBG_ERR_STACK_OVERFLOW = 5, /* traversal stack exceeded its capacity */
    BBG_ERR_CUDA = 6,           /* any other CUDA runtime error */
    BBG_ERR_BAD_BVH = 7,        /* node array failed validation before upload */
    BBG_ERR_UNSUPPORTED = 8,    /* a feature outside this library's scope */
    BBG_ERR_NO_DEVICE = 9       /* no CUDA device of compute capability 10.0 */
} bbg_status;

/* Where the buffers of a call live. HOST buffers are copied to and from the
 * device inside the call; DEVICE buffers are used in place. */
typedef enum bbg_memory
{
    BBG_MEM_HOST = 0,
    BBG_MEM_DEVICE = 1
} bbg_memory;

/* ---------------------------------------------------------------- geometry */

/* One flattened BVH node: byte-for-byte the reference's LinearBVHNode
 * (include/bulbit/bvh.h:46-57): AABB (min xyz, max xyz), then the union of
 * primitives_offset / child2_offset, uint16 primitive_count, uint8 axis. */
typedef struct bbg_bvh_node
{
    float bmin[3];
    float bmax[3];
    int32_t offset;  /* leaf: first slot; interior: index of the second child */
    uint16_t count;  /* leaf: number of primitives; 0 marks an interior node */
    uint8_t axis;    /* interior: split axis */
    uint8_t pad;
} bbg_bvh_node;

/* A flattened tree: nodes in depth-first order (first child at index+1), and
 * for each leaf slot the index of the primitive it holds in the primitive list
 * the tree was built over. */
typedef struct bbg_bvh
{
    int32_t n_nodes;
    const bbg_bvh_node* nodes;
    int32_t n_slots;
    const int32_t* slot_prims;
} bbg_bvh;

/* Sphere with the reference's Transform (position p, unit quaternion q as
 * x,y,z,w, scale s) and radius (include/bulbit/shapes.h:12-31). */
typedef struct bbg_sphere
{
    float p[3];
    float q[4];
    float s[3];
    float radius;
} bbg_sphere;

enum
{
    BBG_PRIM_TRIANGLE = 0,
    BBG_PRIM_SPHERE = 1
};

/* Scene geometry. Vertex attributes are the reference Mesh's world-space
 * arrays (include/bulbit/mesh.h:37-41) concatenated over all meshes. Primitive
 * i of the list (the vector handed to BVH) is a triangle (prim_index[i] =
 * triangle number, its vertices tri_indices[3t..3t+2]) or a sphere
 * (prim_index[i] = sphere number). normals/tangents/uvs may be NULL for a
 * scene that is only ever intersected, never shaded. */
typedef struct bbg_geometry
{
    int32_t n_vertices;
    const float* positions; /* 3 per vertex */
    const float* normals;   /* 3 per vertex or NULL */
    const float* tangents;  /* 3 per vertex or NULL */
    const float* uvs;       /* 2 per vertex or NULL */
    int32_t n_triangles;
    const int32_t* tri_indices; /* 3 per triangle */
    int32_t n_spheres;
    const bbg_sphere* spheres;
    int32_t n_prims;
    const int32_t* prim_kind;  /* BBG_PRIM_* per primitive */
    const int32_t* prim_index; /* per primitive */
} bbg_geometry;

/* A ray query: Ray{o, d} with the [t_min, t_max] interval of
 * Intersectable::Intersect (include/bulbit/intersectable.h:42). 32 bytes. */
typedef struct bbg_ray
{
    float o[3];
    float d[3];
    float t_min;
    float t_max;
} bbg_ray;

/* Closest hit: primitive index in the primitive list (-1 on a miss), the
 * reference's Intersection::t, and the barycentrics (u, v) of a triangle hit. */
typedef struct bbg_hit
{
    int32_t prim;
    float t;
    float u;
    float v;
} bbg_hit;

typedef struct bbg_accel bbg_accel;

/* Builds the reference's 12-bucket binned SAH tree (src/accel/bvh.cpp:56-271)
 * over per-primitive AABBs (6 floats each: min xyz, max xyz), flattened
 * depth-first (src/accel/bvh.cpp:273-297). nodes_out must hold 2*n_prims-1
 * nodes and slot_prims_out n_prims entries. Single-threaded and
 * deterministic: leaves take their slots in depth-first order. */
bbg_status bbg_bvh_build(const float* prim_aabbs, int32_t n_prims, bbg_bvh_node* nodes_out,
                         int32_t* slot_prims_out, int32_t* n_nodes_out);

/* Primitive AABBs exactly as Triangle::GetAABB (src/geometry/triangle.cpp:40)
 * and Sphere::GetAABB (src/geometry/sphere.cpp:30) compute them. */
bbg_status bbg_prim_aabbs(const bbg_geometry* geometry, float* aabbs_out);

/* Uploads geometry and a tree to the current device (every later call on the
 * handle runs on that device, whichever is current then, and restores the
 * caller's current device on return; integrators, guides and batches
 * likewise live on the device current at their creation, an integrator on
 * its accel's). bvh == NULL builds the tree with
 * bbg_bvh_build. The tree is validated (child and slot ranges, no cycles)
 * before upload; it has at least one slot per primitive (the reference's
 * tree exactly one; a primitive may fill several). */
bbg_status bbg_accel_create(const bbg_geometry* geometry, const bbg_bvh* bvh, bbg_accel** out);

/* Uploads geometry with a tree built over split references (early split
 * clipping): triangles whose boxes they fill poorly are split along the
 * longest axis of their box, each part keeping the box of the triangle
 * clipped to it (rounded outward, padded like Triangle::GetAABB), up to
 * budget extra references per primitive (budget in [0, 64]; 0 builds the
 * reference's own tree), then bbg_bvh_build runs over the references. A
 * triangle may sit in several leaves; closest hits agree with BVH::Intersect
 * except between primitives hit at exactly the same t. */
bbg_status bbg_accel_create_split(const bbg_geometry* geometry, float budget, bbg_accel** out);

/* The references bbg_accel_create_split builds over (host only): their boxes
 * (6 floats each) and primitives, at most n_prims * (1 + budget) of them;
 * capacity is the room in the output arrays. */
bbg_status bbg_split_references(const bbg_geometry* geometry, float budget, int32_t capacity, float* aabbs_out,
                                int32_t* prims_out, int32_t* n_out);

/* Uploads geometry and builds the tree on the device: a linear BVH (Morton
 * codes of the primitive boxes' centres, radix sort, the binary radix tree
 * of Karras 2012, bottom-up boxes; one primitive per leaf) in milliseconds
 * where the SAH build (reference BVH::BVH, src/accel/bvh.cpp:8) takes seconds
 * on millions of primitives. The tree differs from the reference's, so closest
 * hits agree with BVH::Intersect except between primitives hit at exactly the
 * same t; the binary radix tree is also collapsed into the 8-wide layout on
 * the device (traversal WIDE by default, ORDERED selectable; no reference
 * node order, no counting, no export). */
bbg_status bbg_accel_create_device_build(const bbg_geometry* geometry, bbg_accel** out);

/* Uploads geometry and builds, on the device, the tree bbg_bvh_build builds
 * on the host: the reference's 12-bucket binned SAH tree
 * (BVH::BuildRecursive / FlattenBVH, src/accel/bvh.cpp:56-297) node for node
 * (same boxes, axes, child offsets and leaf primitives in the same order,
 * leaves in depth-first slot order), in milliseconds instead of the host
 * build's seconds on millions of primitives. One launch per tree level: a
 * block per node of more than 32 primitives, a warp per smaller one; the
 * bucket and cost arithmetic is the reference's, and std::partition's swap
 * order is reproduced by prefix sums. Every traversal mode, counting and
 * bbg_accel_export work as for a host-built tree (export copies the tree
 * from the device). */
bbg_status bbg_accel_create_device_sah(const bbg_geometry* geometry, bbg_accel** out);

/* bbg_accel_create_split built on the device: the references are split on
 * the device (early split clipping with the host splitter's clipping, area
 * and rounding rules, in rounds that each split every reference whose wasted
 * box area lies in the highest occupied power-of-two bin, where the host
 * splits the single largest one at a time; right halves appended in
 * reference order, so the result is deterministic), then the device SAH build
 * of bbg_accel_create_device_sah runs over them. budget in [0, 64]; 0 gives
 * bbg_accel_create_device_sah's tree. The reference set, and so the tree,
 * differs from the host splitter's; closest hits agree with BVH::Intersect
 * except between primitives hit at exactly the same t. No counterpart in the
 * reference renderer. */
bbg_status bbg_accel_create_device_split(const bbg_geometry* geometry, float budget, bbg_accel** out);
bbg_status bbg_accel_destroy(bbg_accel* accel);

/* Root AABB (6 floats), as BVH::GetAABB (src/accel/bvh.cpp:363). */
bbg_status bbg_accel_bounds(const bbg_accel* accel, float* aabb_out);

/* Copies the 8-wide node layout back (24 floats per node, in the node
 * format of bulbit_b200/csrc/dev_geometry.cuh); *n_nodes_out receives the
 * node count, 0 where the layout is not built. nodes_out NULL asks for the
 * count only. No counterpart in the reference, whose tree is binary. */
bbg_status bbg_accel_export_wide8(const bbg_accel* accel, float* nodes_out, int32_t* n_nodes_out);

/* Copies the uploaded tree back: n_nodes nodes and n_slots slot entries. */
bbg_status bbg_accel_export(const bbg_accel* accel, bbg_bvh_node* nodes_out, int32_t* slot_prims_out,
                            int32_t* n_nodes_out, int32_t* n_slots_out);

/* Batched BVH::Intersect: one bbg_hit per ray. stream is a cudaStream_t
 * (NULL = the handle's own stream); the call returns after the results are in
 * hits. Host-memory queries are staged through twelve device slots of up to
 * 2M rays (96 MiB each), allocated by the first host query of that size and
 * kept with the handle, so the copies overlap the traversal. */
bbg_status bbg_intersect(bbg_accel* accel, const bbg_ray* rays, int64_t n, bbg_hit* hits, bbg_memory mem,
                         void* stream);

/* Closest-hit queries for callers that cannot allocate device memory when
 * they trace (allocation forbidden after start-up, a real-time loop, or device
 * memory already held by another allocator). No counterpart in the reference:
 * it exists only for such callers. rays and hits are host buffers; at most
 * 262,144 rays per call (larger n returns BBG_ERR_INVALID_ARG). The rays and
 * hits are staged through one fixed device array of about 12 MiB that every
 * device holds, from the first accel created on it until the process exits;
 * the call itself allocates nothing. Set-up happens when an accel is created:
 * the array's address is looked up on that device (this loads the array) and
 * the query's kernels are loaded, so calls do no set-up of their own. All
 * calls share the array: calls that overlap on the GPU (from several threads
 * or handles at once) race and must be serialised by the caller. Results
 * equal bbg_intersect's for the same accel and traversal mode (a counting
 * accel traverses in the reference's order, as bbg_intersect does, but this
 * query records no counts). The library does not support cudaDeviceReset
 * while any of its handles exist. */
bbg_status bbg_intersect_static(bbg_accel* accel, const bbg_ray* rays, int64_t n, bbg_hit* hits);

/* Batched BVH::IntersectAny: occluded[i] = 1 if ray i hits anything in
 * [t_min, t_max]. */
bbg_status bbg_intersect_any(bbg_accel* accel, const bbg_ray* rays, int64_t n, uint8_t* occluded,
                             bbg_memory mem, void* stream);

/* bbg_intersect and bbg_intersect_any that return once the query is queued;
 * the results are in place after bbg_accel_synchronize (or after any
 * synchronous query on the same accel, which first waits for the submitted
 * ones). Submitted host-memory queries chain through the accel's staging:
 * the copy in of the next query's rays overlaps the traversal of the one
 * before it, so a closest-hit batch and an any-hit batch submitted back to
 * back cost about their copies, not copies plus traversals. Host buffers
 * must stay valid and unchanged until then; in page-locked memory
 * (cudaHostAlloc / cudaHostRegister) the call returns before the copies
 * run, from pageable memory the copies of results block the caller as the
 * synchronous call does. A host batch larger than every earlier one on the
 * handle (below 2M rays) regrows the staging and so first waits for the
 * queued work. Device buffers are traced on the handle's stream.
 * Results equal the synchronous calls'. A counting accel
 * (bbg_accel_set_counting) refuses them (BBG_ERR_UNSUPPORTED). Errors of the
 * queued work are returned by bbg_accel_synchronize. No counterpart in the
 * reference, whose queries are per ray. */
bbg_status bbg_intersect_submit(bbg_accel* accel, const bbg_ray* rays, int64_t n, bbg_hit* hits, bbg_memory mem);
bbg_status bbg_intersect_any_submit(bbg_accel* accel, const bbg_ray* rays, int64_t n, uint8_t* occluded,
                                    bbg_memory mem);
bbg_status bbg_accel_synchronize(bbg_accel* accel);

/* Traversal order. WIDE (the default) traverses the tree collapsed into
 * 8-wide nodes with byte-quantised child boxes (rounded outward), children
 * ordered by ray octant; ORDERED (the default where the 8-wide layout cannot
 * be built) visits the nearer child first over a binary child-box node
 * layout and skips subtrees beyond the closest hit so far; REFERENCE visits
 * nodes in BVH::RayCast's own order (include/bulbit/bvh.h:102-155; not for
 * trees built on the device). All run the same
 * primitive tests and return the same closest primitive and t; they can
 * differ only on rays whose two nearest hits have exactly equal t (the
 * reference keeps the last one it visits). Any-hit results are identical.
 * The choice also applies to renders with the accel. */
enum
{
    BBG_TRAVERSAL_ORDERED = 0,
    BBG_TRAVERSAL_REFERENCE = 1,
    BBG_TRAVERSAL_WIDE = 2
};
bbg_status bbg_accel_set_traversal(bbg_accel* accel, int32_t mode);

/* Traversal statistics of the last bbg_intersect / bbg_intersect_any call on
 * this handle when counting is enabled: nodes popped and slab-tested, and
 * primitive tests, summed over all rays, for a traversal in the reference's
 * node order (a counting call always uses that order). */
bbg_status bbg_accel_set_counting(bbg_accel* accel, int32_t enable);
bbg_status bbg_accel_last_counts(const bbg_accel* accel, int64_t* nodes_visited, int64_t* prims_tested);

/* ---------------------------------------------------------------- shading */

enum
{
    BBG_MAT_NONE = -1,
    BBG_MAT_DIFFUSE = 0,            /* DiffuseMaterial, roughness 0: LambertianBxDF */
    BBG_MAT_CONDUCTOR = 1,          /* ConductorMaterial */
    BBG_MAT_DIELECTRIC = 2,         /* DielectricMaterial */
    BBG_MAT_METALLIC_ROUGHNESS = 3  /* MetallicRoughnessMaterial */
};

/* Constant-texture material parameters.
 *   DIFFUSE:   reflectance = albedo
 *   CONDUCTOR: eta, k (RGB); reflectance = lobe reflectance (1,1,1 default);
 *              conductor_from_r != 0 selects the (R, roughness) constructor,
 *              with R in k (include/bulbit/bxdfs.h:261-272)
 *   DIELECTRIC: eta[0] = index of refraction; reflectance = reflectance
 *   METALLIC_ROUGHNESS: reflectance = basecolor, metallic
 *   roughness[0], roughness[1] = u and v roughness (alpha = roughness^2, or
 *   max(roughness^2, 1e-3) for METALLIC_ROUGHNESS). */
typedef struct bbg_material
{
    int32_t type;
    int32_t conductor_from_r;
    float reflectance[3];
    float eta[3];
    float k[3];
    float roughness[2];
    float metallic;
    int32_t energy_compensation; /* CONDUCTOR / DIELECTRIC: the material's
                                    energy_compensation (ConductorMultiScatteringBxDF /
                                    DielectricMultiScatteringBxDF: a multiple-
                                    scattering lobe from the energy tables) */
} bbg_material;

enum
{
    BBG_LIGHT_POINT = 0,
    BBG_LIGHT_SPOT = 1,
    BBG_LIGHT_UNIFORM_INFINITE = 2,
    BBG_LIGHT_DIFFUSE_AREA = 3
};

/* Light parameters, as the reference constructors take them
 * (include/bulbit/lights.h):
 *   POINT:  position, intensity
 *   SPOT:   position, direction (the ctor's "direction" argument), intensity,
 *           angle_max / angle_falloff_start in degrees
 *   UNIFORM_INFINITE: intensity = L, scale
 *   DIFFUSE_AREA: prim (primitive index), intensity = constant emission,
 *           two_sided */
typedef struct bbg_light
{
    int32_t type;
    int32_t prim;
    int32_t two_sided;
    float position[3];
    float direction[3];
    float intensity[3];
    float scale;
    float angle_max;
    float angle_falloff_start;
} bbg_light;

/* PerspectiveCamera inputs (src/camera/perspective_camera.cpp:8) with a
 * Transform::LookAt(position, target, up) pose and a BoxFilter(extent). */
/* Reconstruction filters (src/reconstruction/{box,tent,gaussian}_filter.cpp):
 * the filter's Sample(u) places each camera sample in its pixel. */
enum
{
    BBG_FILTER_BOX = 0,
    BBG_FILTER_TENT = 1,
    BBG_FILTER_GAUSSIAN = 2
};

typedef struct bbg_camera_spec
{
    float position[3];
    float target[3];
    float up[3];
    float vfov_deg;
    float aperture_radius;
    float focus_distance;
    int32_t width;
    int32_t height;
    float filter_extent;
    int32_t filter_type;  /* BBG_FILTER_* (0: box) */
    float filter_sigma;   /* Gaussian standard deviation (GaussianFilter(sigma, extent)) */
} bbg_camera_spec;

/* The derived state PerspectiveCamera::SampleRay reads
 * (include/bulbit/cameras.h:50-61). */
typedef struct bbg_camera
{
    int32_t width;
    int32_t height;
    float origin[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
    float u[3];
    float v[3];
    float lens_radius;
    float filter_extent;
    int32_t filter_type;
    float filter_sigma;
} bbg_camera;

bbg_status bbg_camera_perspective(const bbg_camera_spec* spec, bbg_camera* out);

typedef struct bbg_integrator bbg_integrator;

/* PathIntegrator(accel, lights, sampler, max_bounces, rr_min_bounces,
 * regularize_bsdf) with a PowerLightSampler. prim_material[i] is the material
 * index of primitive i or BBG_MAT_NONE (a medium boundary: rays pass
 * through). Lights are preprocessed against the accel's bounds as the
 * reference Integrator constructor does. */
bbg_status bbg_integrator_create(bbg_accel* accel, const int32_t* prim_material, const bbg_material* materials,
                                 int32_t n_materials, const bbg_light* lights, int32_t n_lights,
                                 int32_t max_bounces, int32_t rr_min_bounces, int32_t regularize_bsdf,
                                 bbg_integrator** out);
bbg_status bbg_integrator_destroy(bbg_integrator* integrator);

/* Light selection pmf of each light (PowerLightSampler::EvaluatePMF,
 * src/light_sampler/power_light_sampler.cpp:44). */
bbg_status bbg_integrator_light_pmf(const bbg_integrator* integrator, float* pmf_out);

typedef struct bbg_render_params
{
    int32_t spp;          /* IndependentSampler samples_per_pixel */
    int32_t seed;         /* IndependentSampler seed */
    int64_t wave_paths;   /* paths in flight per wave; 0 = library default */
    int32_t use_graph;    /* capture the bounce loop of a wave in a CUDA graph */
    int32_t light_alias;  /* 1: sample lights with a Walker alias table (same
                             pmf, different stream) instead of CDF inversion */
    struct bbg_guide* guide; /* NULL: the reference's estimator. Otherwise, at
                                non-specular vertices, one-sample MIS between
                                the guide and the BSDF (a different random
                                stream, same expectation) */
    int32_t guide_train;  /* 1: train the guide online on this render's paths,
                             one Adam step per wave */
    int32_t guide_batch;  /* training samples per step (0: 65536) */
    float guide_lr;       /* Adam learning rate (0: 1e-2) */
    float guide_select;   /* probability of sampling the guide rather than the
                             BSDF, in (0, 1] (0: 1/2) */
    int32_t guide_steps;  /* Adam steps per wave when training, each on its own
                             batch of guide_batch training samples (0: 1) */
    int32_t sampler;      /* BBG_SAMPLER_INDEPENDENT (0) or BBG_SAMPLER_STRATIFIED:
                             StratifiedSampler(x_samples, spp / x_samples, jitter,
                             seed), src/sampler/stratified_sampler.cpp */
    int32_t x_samples;    /* stratified: strata along x (spp must be a multiple) */
    int32_t jitter;       /* stratified: jitter within strata */
    int32_t shade_order;  /* BBG_SHADE_SORTED (0): each bounce level's paths are
                             shaded grouped by material kind (a counting sort
                             of the level's queue); BBG_SHADE_QUEUE: in queue
                             order. Results are identical; guided renders shade
                             in queue order. */
    int32_t pass_through_levels; /* paths that cross material-less surfaces
                             (which count no bounce) may outlive the
                             max_bounces + 1 levels of a wave; they are traced
                             on, level by level, for at most this many extra
                             levels (0: 4096) before the render gives up with
                             BBG_ERR_TIMEOUT */
} bbg_render_params;

enum
{
    BBG_SAMPLER_INDEPENDENT = 0,
    BBG_SAMPLER_STRATIFIED = 1
};

enum
{
    BBG_SHADE_SORTED = 0,
    BBG_SHADE_QUEUE = 1
};

/* Per-pixel film state, W*H entries each, pixel index y*W + x. The fields
 * are those Film::AddSample maintains (src/reconstruction/film.cpp:26-37):
 * radiance sum, sample count (NaN/Inf samples are skipped), and luminance
 * moments. path_L, if not NULL, receives each path's radiance (3 floats per
 * path, path index (y*W + x)*spp + sample). */
typedef struct bbg_film
{
    float* rgb_sum;
    int32_t* count;
    float* moments;
    float* path_L;
} bbg_film;

typedef struct bbg_render_stats
{
    int64_t paths;
    int64_t closest_rays;   /* closest-hit rays traced */
    int64_t shadow_rays;    /* shadow rays traced */
    double device_ms;       /* device time of the render's waves, CUDA events
                               (buffer set-up and graph capture, once per
                               configuration, excluded) */
} bbg_render_stats;

bbg_status bbg_render(bbg_integrator* integrator, const bbg_camera* camera, const bbg_render_params* params,
                      bbg_film* film, bbg_memory mem, bbg_render_stats* stats);

/* --------------------------------------------------- batches of scenes */

/* Several scenes rendered together (no counterpart in the reference, whose
 * Render() takes one scene). Each stage of the wavefront — ray generation,
 * closest hit, shading, shadow rays, film — runs once per bounce level over
 * the paths of all scenes: every path is traced in its own scene's tree and
 * shaded with its own materials and lights, so scenes of very different
 * sizes share the GPU instead of leaving it idle in turn. Every path keeps
 * the sampler stream and arithmetic of its scene's own bbg_render, so each
 * scene's film equals rendering that scene alone. */
typedef struct bbg_batch bbg_batch;

bbg_status bbg_batch_create(bbg_batch** out);
bbg_status bbg_batch_destroy(bbg_batch* batch);
/* Renders n scenes (1 <= n <= 2048): integrators[i] seen through cameras[i]
 * with params[i] into films[i] (host or device memory as mem says). Every
 * params[i].spp must be equal; every accel must use an ordered traversal
 * (WIDE or ORDERED; the 8-wide layout is traversed when every accel selects
 * it). The wave size and CUDA-graph choice come from params[0].
 * Guided batches: either every params[i].guide is set (a distinct guide per
 * scene, n <= 64) or none is. Each bounce level then buckets the guide
 * queries by scene and runs all scenes' MLPs in one grouped forward launch
 * (each 128-query chunk with its scene's weights); with guide_train, each
 * scene's guide is trained on that scene's records of the wave. The guide
 * settings (train, batch, steps, lr, select) come from params[0].
 * stats (optional) receives the batch's totals.
 * Calls on one batch must not overlap, nor overlap renders of the same
 * integrators (their film buffers are reused for host-memory films). */
bbg_status bbg_batch_render(bbg_batch* batch, int32_t n, bbg_integrator* const* integrators,
                            const bbg_camera* cameras, const bbg_render_params* params, bbg_film* films,
                            bbg_memory mem, bbg_render_stats* stats);

/* The GGX energy tables the energy-compensated conductor uses, as the
 * reference computes them (TrowbridgeReitzDistribution::
 * PrepareReflectanceTexture, src/bxdf/microfacet.cpp:28-70; samples from
 * PrepareReflectanceTextures, :239-275): e_out 32 x 32 (index cos_i + 32 *
 * alpha_j), e_avg_out 32. Computed on the device once per process. */
bbg_status bbg_ggx_energy_tables(float* e_out, float* e_avg_out);

/* The rough-dielectric energy tables the energy-compensated dielectric uses
 * (DielectricMultiScatteringBxDF::PrepareReflectanceTexture,
 * src/bxdf/microfacet.cpp:168-237): e_out and e_inv_out 32 x 32 x 32 (index
 * f0_k + 32 * (cos_i + 32 * alpha_j); e for eta >= 1, e_inv for the inverse
 * interface), e_avg_out and e_inv_avg_out 32 x 32 (index f0_k + 32 *
 * alpha_j). Computed on the device once per process. */
bbg_status bbg_dielectric_energy_tables(float* e_out, float* e_inv_out, float* e_avg_out, float* e_inv_avg_out);

/* ------------------------------------------------------------ autotuning */

/* Launch configuration of a render: the traversal passes' threads per block
 * and traversal-stack entries per thread kept in shared memory (0: the whole
 * stack in local memory), and the wave size (paths in flight, which sizes
 * every queue). No counterpart in the reference. */
typedef struct bbg_tuning
{
    int32_t block;        /* 128 or 256 */
    int32_t short_stack;  /* 0, 8 or 16 (16 only with block 128 or 256) */
    int64_t wave_paths;
    double probe_ms;      /* device time per million paths of the chosen probe */
    int32_t from_cache;   /* 1: reused from an identical scene, nothing timed */
} bbg_tuning;

/* Chooses the configuration for renders of this scene, camera size, spp and
 * bounce limit by timing short probe renders (first each launch shape at the
 * default wave size, then each wave size from 2^20 to 2^26 paths that the
 * render can fill and whose path state, about 157 bytes per path, fits in a
 * quarter of the free device memory), keeps it for the integrator's later renders that leave
 * wave_paths at 0, and caches it per scene signature (primitive and node
 * counts, tree depth, image size, spp, bounces) for the process, so a later
 * identical scene is not timed again. params: spp and seed of the renders to
 * tune for (guide must be NULL). */
bbg_status bbg_integrator_autotune(bbg_integrator* integrator, const bbg_camera* camera,
                                   const bbg_render_params* params, bbg_tuning* out);
/* Sets the configuration directly (block/short_stack must be one of the
 * combinations above; wave_paths 0 = default). */
bbg_status bbg_integrator_set_tuning(bbg_integrator* integrator, const bbg_tuning* tuning);
/* The same for a batch of scenes (the arguments of bbg_batch_render). */
bbg_status bbg_batch_autotune(bbg_batch* batch, int32_t n, bbg_integrator* const* integrators,
                              const bbg_camera* cameras, const bbg_render_params* params, bbg_tuning* out);

/* The first n uniform draws of IndependentSampler after
 * StartPixelSample(pixel, sample) with the given seed, computed on the device. */
bbg_status bbg_sampler_draws(int32_t px, int32_t py, int32_t seed, int32_t sample, int32_t n, float* out);

/* Material::GetBSDF (the src/material sources) at a surface with shading normal +z
 * and tangent +x (local = world directions; front_face selects the
 * dielectric's relative eta), then BSDF::f, PDF and Sample_f
 * (include/bulbit/bsdf.h:73-125) for n queries (wo, wi, u: 3 floats each).
 * out: 12 floats per query — f (rgb), pdf, the sample's f (rgb), wi, pdf and
 * flags (-1 where Sample_f fails). */
bbg_status bbg_bsdf_probe(const bbg_material* material, int32_t front_face, int32_t n, const float* wo,
                          const float* wi, const float* u, float* out);

/* --------------------------------------------------------- path guiding */

/* Neural path guiding (no counterpart in the reference: an added learned
 * component). A small MLP maps a shading point — raw query of 10 floats:
 * position (3), shading normal (3), outgoing direction (3), roughness — to an
 * 8-lobe von Mises-Fisher mixture over incident directions (40 outputs: per
 * lobe weight logit, unnormalised mean (3), log kappa). Network 80 -> 64 ->
 * 64 -> 64 -> 40 (ReLU), 16,104 parameters; BF16 weights and activations on
 * the tensor cores, FP32 accumulation and FP32 master weights; Adam
 * (betas 0.9 / 0.99). The position is normalised by scene_aabb (min xyz,
 * max xyz). Host buffers throughout. */
typedef struct bbg_guide bbg_guide;

bbg_status bbg_guide_create(const float* scene_aabb, uint64_t seed, bbg_guide** out);
bbg_status bbg_guide_destroy(bbg_guide* guide);
/* FP32 master parameters, 16,104 floats: W0 b0 W1 b1 W2 b2 W3 b3, W [out][in]. */
bbg_status bbg_guide_get_params(bbg_guide* guide, float* params_out);
bbg_status bbg_guide_set_params(bbg_guide* guide, const float* params);
/* Network outputs (40 per query) for n raw queries. */
bbg_status bbg_guide_forward(bbg_guide* guide, const float* raw, int64_t n, float* out);
/* Gradient (16,104 floats) of sum_i -weights[i] * log q_i(dirs[i]) over n
 * samples (dirs: 3 floats each, unit length), and that sum in *loss_out. */
bbg_status bbg_guide_gradient(bbg_guide* guide, const float* raw, const float* dirs, const float* weights, int64_t n,
                              float* grad_out, float* loss_out);
/* One Adam step on the mean of that loss over the batch; *loss_out = mean loss
 * before the step. */
bbg_status bbg_guide_train_step(bbg_guide* guide, const float* raw, const float* dirs, const float* weights, int64_t n,
                                float learning_rate, float* loss_out);

/* The vMF mixture a network output row describes (40 floats), evaluated on
 * the device exactly as the guided renderer does: sample n directions with
 * uniforms u (3 per row; pdf_out receives the mixture density of each), or
 * evaluate the density at n unit directions. Host buffers. */
bbg_status bbg_guide_mixture_sample(const float* outputs, const float* u, int64_t n, float* dirs_out, float* pdf_out);
bbg_status bbg_guide_mixture_pdf(const float* outputs, const float* dirs, int64_t n, float* pdf_out);

/* --------------------------------------------------------------- library */

const char* bbg_last_error(void);
const char* bbg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BBG_H */
