// The guide handle (neural path guiding) and its launch helpers.
#pragma once

#include "cuda_util.cuh"
#include "dev_guide.cuh"

struct bbg_guide
{
    int device = 0; // the device that was current at creation; every call runs there
    cudaStream_t stream = nullptr;
    bbg::GuideBounds bounds{};
    bbg::DevBuf<float> params;  // FP32 master parameters (kGuideParams)
    bbg::DevBuf<float> adam_m, adam_v, grad, loss;
    bbg::DevBuf<__nv_bfloat16> bf16; // kBfBuf: training forward + transposed + tensor-core forward images
    bbg::DevBuf<int32_t> step_dev; // Adam step counter
    bbg::DevBuf<__nv_bfloat16> scratch; // training: transposed activations and gradients
    bbg::DevBuf<float> partial;         // training: per-chunk weight-gradient partial sums
    bbg::DevBuf<int32_t> tc_status;     // nonzero: a tensor-core pass (forward or weight gradients) timed out
    float beta1 = 0.9f, beta2 = 0.99f;
    bool smem_set = false;
    // Staging for host-buffer calls.
    bbg::DevBuf<float> s_raw, s_dirs, s_w, s_out;

    ~bbg_guide()
    {
        if (stream)
        {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

namespace bbg
{
// Queries per chunk of the grouped forward (one 128-query tensor-core tile):
// each group's queries start on a chunk boundary, so a chunk reads one
// group's weights.
constexpr int kGuideGroupChunk = 128;

// One group's guide as the grouped forward reads it (the device addresses
// of its BF16 weight images, FP32 parameters and time-out status, and its
// scene bounds).
struct GuideGroup
{
    const __nv_bfloat16* wg;
    const float* pg;
    int32_t* status;
    GuideBounds bounds;
};

// Sets the kernels' shared-memory limits (once) and returns the forward grid.
bbg_status GuidePrepare(bbg_guide* G, int* grid);
// Forward over n queries (raw records of kGuideRaw floats); index (optional)
// maps query i to record index[i] for both raw and out. n from n_dev if set.
bbg_status GuideForward(bbg_guide* G, const float* raw_dev, const int32_t* index_dev, const int32_t* n_dev,
                        int64_t n_host, float* out_dev, cudaStream_t st);
// Forward over queries bucketed by group (grouped BF16 GEMMs in one launch):
// index_dev lists record indices, group g's from chunk chunk_start_dev[g] to
// chunk_start_dev[g + 1] (kGuideGroupChunk entries each, -1 for padding);
// groups_dev[g] holds group g's guide. Output per record, as GuideForward.
bbg_status GuideForwardGrouped(const float* raw_dev, const int32_t* index_dev, const int32_t* chunk_start_dev,
                               int32_t n_groups, const GuideGroup* groups_dev, float* out_dev, cudaStream_t st);
// Allocates the training scratch for batches of up to capacity samples (so
// that no allocation falls inside a timed or captured render).
bbg_status GuideReserveTraining(bbg_guide* G, int64_t capacity);
// Adds the gradient of sum_i -w_i log q_i(dir_i) to the guide's accumulator;
// capacity bounds n (n from n_dev if set) and sizes the training scratch.
bbg_status GuideAccumulate(bbg_guide* G, const float* raw_dev, const float* dirs_dev, const float* weights_dev,
                           const int32_t* n_dev, int64_t n_host, int64_t capacity, cudaStream_t st);
// BBG_ERR_TIMEOUT if a forward or weight-gradient pass of this guide has
// given up waiting for its tensor-core MMAs (synchronises with the device).
bbg_status GuideCheckStatus(bbg_guide* G);
// One Adam step with gradient = accumulator / n (n from n_dev if set); an
// empty batch is skipped.
bbg_status GuideApply(bbg_guide* G, float lr, const int32_t* n_dev, int64_t n_host, cudaStream_t st);
} // namespace bbg
