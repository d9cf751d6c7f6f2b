// The accel handle: geometry and flattened BVH resident on the device.
#pragma once

#include "cuda_util.cuh"
#include "dev_geometry.cuh"

#include <vector>

struct bbg_accel
{
    int device = 0; // the device that was current at creation; every call runs there
    cudaStream_t stream = nullptr;
    int32_t n_prims = 0;
    int32_t n_nodes = 0;
    int32_t n_slots = 0;
    int32_t max_depth = 0;
    float bounds[6] = {};

    // Traversal data.
    bbg::DevBuf<float4> nodes; // 2 float4 per node
    bbg::DevBuf<float4> slots; // 3 float4 per slot
    bbg::DevBuf<float4> wide;  // 4 float4 per interior node (child-box layout)
    bbg::DevBuf<int2> leaves;  // (first slot, count) per leaf
    int32_t root = 0;
    bool ordered = true;
    bbg::DevBuf<float4> wide8; // 6 float4 per node (8-wide layout; empty if not built)
    int32_t root8 = 0;
    int32_t n_wide8 = 0;
    int32_t depth8 = 0;
    bool use_wide8 = false;    // ordered queries run over the 8-wide layout
    bool device_built = false; // linear BVH built on the device (no reference node layout)
    bool device_sah = false;   // the reference's SAH tree built on the device (tree arrays device-only)
    bbg::DevBuf<int32_t> slot_prims; // device_sah: slot -> primitive (for export)

    // Shading data (the reference Mesh arrays and shapes).
    bbg::DevBuf<int2> prim_shape;     // (kind, index) per primitive
    bbg::DevBuf<int32_t> tri_indices; // 3 per triangle
    bbg::DevBuf<float> positions;     // 3 per vertex
    bbg::DevBuf<float> normals;       // 3 per vertex
    bbg::DevBuf<float> tangents;      // 3 per vertex
    bbg::DevBuf<float> uvs;           // 2 per vertex
    bbg::DevBuf<bbg_sphere> spheres;
    bool has_shading = false;
    bool has_spheres = false; // any sphere primitive (else the triangle-only traversal kernels run)

    // Host copies of the tree (export, light set-up).
    std::vector<bbg_bvh_node> host_nodes;
    std::vector<int32_t> host_slots;
    std::vector<int2> host_prim_shape;
    std::vector<int32_t> host_tri_indices;
    std::vector<float> host_positions;
    std::vector<bbg_sphere> host_spheres;

    // Staging for host-memory calls: a ring of kHostStages slots; rays go in
    // on copy_stream[0], the kernels run on `stream`, results come back on
    // copy_stream[1], ordered by per-slot events. The ring position carries
    // over from call to call, so submitted queries chain through it. Twelve
    // slots of up to 2M rays let the copy in run eleven chunks ahead of the
    // traversal, also where the chunks are short (a batch's ramp down and the
    // next one's ramp up): through a closest-hit batch, whose traversal is
    // slower than its copy, into the next batch's rays.
    static constexpr int kHostStages = 12;
    bbg::DevBuf<float4> stage_in[kHostStages];
    bbg::DevBuf<float4> stage_out[kHostStages];
    cudaStream_t copy_stream[2] = { nullptr, nullptr };
    cudaEvent_t ev_in[kHostStages] = {};     // slot's rays copied in
    cudaEvent_t ev_traced[kHostStages] = {}; // slot's rays traced (stage_in free)
    cudaEvent_t ev_out[kHostStages] = {};    // slot's results copied out (stage_out free)
    int stage_next = 0;                      // ring slot of the next chunk
    bool pending = false;                    // submitted queries not yet synchronised

    // Traversal counters (nodes, prims) of the last call when enabled.
    bool counting = false;
    bbg::DevBuf<unsigned long long> counters;
    bbg::DevBuf<int32_t> work; // persistent-kernel work counter
    int64_t last_nodes = 0, last_prims = 0;

    bbg::AccelView view() const
    {
        return bbg::AccelView{ nodes.p, slots.p, wide.p, leaves.p, root, ordered ? 1 : 0, wide8.p, root8 };
    }
    bool wide8_active() const { return ordered && use_wide8 && wide8.p != nullptr; }
};

namespace bbg
{
// Launches the batched traversal kernel on device-resident rays.
bbg_status LaunchIntersect(bbg_accel* a, const float4* rays, int64_t n, float4* hits, cudaStream_t stream);
bbg_status LaunchIntersectAny(bbg_accel* a, const float4* rays, int64_t n, uint8_t* occluded, cudaStream_t stream);
// Builds a linear BVH on the device (lbvh.cu) over the uploaded geometry:
// fills slots, the child-box layout, leaves, root, bounds and depth.
bbg_status BuildLbvh(bbg_accel* a, const bbg_geometry* g);
// Builds the reference's binned SAH tree on the device (sah_build.cu), node
// for node as BuildBvh does on the host, over n items of the uploaded
// geometry: its primitives (ref_box null) or references (boxes, two float4
// corners each, and the primitive each one belongs to). Fills the reference
// nodes, slots, the child-box layout, leaves, root, the 8-wide layout,
// bounds, depth and the slot primitives.
bbg_status BuildSahOnDevice(bbg_accel* a, int32_t n, const float4* ref_box, const int32_t* ref_prim);
// References for a tree over split primitives (early split clipping), made
// on the device: at most n_prims * (1 + budget) of them, their boxes and
// primitives; *n_refs receives the count.
bbg_status SplitReferencesOnDevice(bbg_accel* a, float budget, DevBuf<float4>* ref_box, DevBuf<int32_t>* ref_prim,
                                   int32_t* n_refs);
// Looks up (once per device, the current one) the device address of the
// allocation-free query's fixed array, which also makes the array exist on
// that device from this point until the process exits (noalloc.cu).
bbg_status ReserveStaticScratch();
} // namespace bbg
