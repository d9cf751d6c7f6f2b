// Small CUDA helpers: status-returning error checks and owning device buffers.
#pragma once

#include "bbg_internal.h"

#include <cuda_runtime.h>
#include <utility>

namespace bbg
{

#define BBG_CUDA(call)                                                                                                 \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess)                                                                                         \
        {                                                                                                              \
            return ::bbg::Fail(e_ == cudaErrorMemoryAllocation ? BBG_ERR_OOM : BBG_ERR_CUDA, "%s failed: %s", #call,  \
                               cudaGetErrorString(e_));                                                                \
        }                                                                                                              \
    } while (0)

#define BBG_TRY(expr)                                                                                                  \
    do                                                                                                                 \
    {                                                                                                                  \
        bbg_status s_ = (expr);                                                                                        \
        if (s_ != BBG_OK)                                                                                              \
        {                                                                                                              \
            return s_;                                                                                                 \
        }                                                                                                              \
    } while (0)

template <typename T>
struct DevBuf
{
    T* p = nullptr;
    size_t n = 0;

    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }

    void reset()
    {
        if (p)
        {
            cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }

    bbg_status alloc(size_t count)
    {
        if (count <= n && p)
        {
            return BBG_OK;
        }
        reset();
        if (count == 0)
        {
            return BBG_OK;
        }
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
        if (e != cudaSuccess)
        {
            p = nullptr;
            return Fail(BBG_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        n = count;
        return BBG_OK;
    }

    bbg_status upload(const T* host, size_t count, cudaStream_t stream = 0)
    {
        BBG_TRY(alloc(count));
        if (count)
        {
            BBG_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        }
        return BBG_OK;
    }
};

// The current device must be a compute-capability 10.x part (the kernels are
// sm_100a).
bbg_status CheckDevice();

// Grid size for a grid-stride kernel on the current device: resident blocks
// per SM x SM count.
int PersistentGrid(const void* kernel, int block, size_t smem = 0);

// SM count of the current device.
int CurrentSmCount();

// Makes `device` current for the scope of a call on a handle and restores the
// caller's current device on exit. Handles remember the device that was
// current when they were created; every later call on them runs there, so
// one process can hold handles on several GPUs.
class DeviceScope
{
public:
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device)
        {
            ok_ = cudaSetDevice(device) == cudaSuccess;
            switched_ = ok_;
        }
    }
    ~DeviceScope()
    {
        if (switched_)
        {
            cudaSetDevice(prev_);
        }
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    bool ok() const { return ok_; }

private:
    int prev_ = -1;
    bool switched_ = false;
    bool ok_ = true;
};

} // namespace bbg
