// Host-side internals shared by the library's translation units: device
// buffers, error propagation and the built acceleration structure.
#pragma once

#include "../../include/colvillea_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace clb
{
// Host milliseconds this thread has spent in cudaMalloc (the allocation share
// of a build's wall time).
double& allocMs();

// Device allocation owned by one object (the reference's DeviceBuffer,
// src/core/devices/cudabuffer.h:39-96, with errors returned, not exit()).
struct DevBuf
{
    void*  p     = nullptr;
    size_t bytes = 0;
    DevBuf()     = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p     = nullptr;
        bytes = 0;
    }
    cl_status alloc(size_t n, std::string* err)
    {
        release();
        if (n == 0) n = 16;
        const auto  t0 = std::chrono::steady_clock::now();
        cudaError_t e  = cudaMalloc(&p, n);
        allocMs() += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (e != cudaSuccess)
        {
            p    = nullptr;
            *err = std::string("cudaMalloc(") + std::to_string(n) + ") failed: " + cudaGetErrorString(e);
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? CL_ERR_OOM : CL_ERR_CUDA;
        }
        bytes = n;
        return CL_OK;
    }
    float*    f() const { return static_cast<float*>(p); }
    uint32_t* u() const { return static_cast<uint32_t*>(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

#define CL_TRY(expr)                                                                                                   \
    do                                                                                                                 \
    {                                                                                                                  \
        cl_status _s = (expr);                                                                                         \
        if (_s != CL_OK) return _s;                                                                                    \
    } while (0)

#define CL_CUDA(expr, errp)                                                                                            \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t _e = (expr);                                                                                       \
        if (_e != cudaSuccess)                                                                                         \
        {                                                                                                              \
            *(errp) = std::string(#expr) + ": " + cudaGetErrorString(_e);                                              \
            return CL_ERR_CUDA;                                                                                        \
        }                                                                                                              \
    } while (0)

struct WideBvh
{
    DevBuf   nodes; // 5 uint4 per node
    DevBuf   tris;  // 3 float4 per triangle, leaf order
    DevBuf   exact; // refit: 6 floats per node, the unquantised box of its triangles
    DevBuf   scene; // scene bounds (6 ordered ints, refit) and the SAH sum (double at byte 32)
    // Nodes of tree level d are [levels[d], levels[d + 1]): the collapse
    // allocates each level's nodes in one launch.
    std::vector<uint32_t> levels;
    uint32_t numNodes = 0, depth = 0, numTris = 0, buildIterations = 0;
    void     release()
    {
        nodes.release();
        tris.release();
        exact.release();
        scene.release();
        levels.clear();
        numNodes = depth = numTris = 0;
    }
};

// A builder temporary: device memory taken from a build arena, with DevBuf's
// accessors; it owns nothing (release() is a no-op).
struct ScratchBuf
{
    void*  p     = nullptr;
    size_t bytes = 0;
    void      release() {}
    float*    f() const { return static_cast<float*>(p); }
    uint32_t* u() const { return static_cast<uint32_t*>(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Grow-only device memory for the builder's temporaries: the k-th temporary of
// a build reuses the k-th block of the previous build that shared the arena
// (growing it when too small), so a sequence of builds (one per mesh of a
// two-level scene) allocates, and frees - a synchronising cudaFree - once.
class BuildArena
{
public:
    void      reset() { used_ = 0; }
    cl_status take(ScratchBuf& s, size_t bytes, std::string* err)
    {
        if (used_ == blocks_.size()) blocks_.emplace_back(new DevBuf());
        DevBuf& b = *blocks_[used_++];
        if (b.bytes < bytes) CL_TRY(b.alloc(bytes, err));
        s.p     = b.p;
        s.bytes = bytes;
        return CL_OK;
    }
    // Device copy of a build's input, kept apart from the temporaries (which
    // reset() recycles): one block that grows and is reused by the next build.
    cl_status input(ScratchBuf& s, size_t bytes, std::string* err)
    {
        if (input_.bytes < bytes) CL_TRY(input_.alloc(bytes, err));
        s.p     = input_.p;
        s.bytes = bytes;
        return CL_OK;
    }

private:
    std::vector<std::unique_ptr<DevBuf>> blocks_;
    size_t                               used_ = 0;
    DevBuf                               input_;
};

// dTri9: 9 floats per triangle (world-space vertices), device memory.  The
// builder's temporaries come from `arena` (a local one when null).
cl_status buildWideBvh(const float* dTri9, uint32_t n, cudaStream_t st, WideBvh* out, std::string* err,
                       BuildArena* arena = nullptr);

// Refit after the vertices moved (same triangles, same vertex indices):
// rewrites the leaf triangles from vtx (3 float4 per vertex, position in the
// first) and triIdx (uint4 per triangle), then recomputes every node's child
// boxes level by level from the deepest, keeping the tree's topology and
// slot order.  Without moved vertices the nodes come out bit-identical to the
// build's.  Asynchronous on st.
cl_status refitWideBvh(WideBvh* bvh, const void* vtx, const void* triIdx, cudaStream_t st, std::string* err);

// Surface-area cost of the built tree: sum over child slots of the slot's
// quantised box area, times the triangle count for leaf slots, over the root
// box area (one unit per node visit and per triangle test).  Synchronises st.
cl_status wideBvhSahCost(WideBvh& bvh, cudaStream_t st, double* cost, std::string* err);

// Triangle positions (9 floats each, triangle order) gathered from vtx and
// triIdx, the input of buildWideBvh.  Asynchronous on st.
cl_status gatherTrianglePositions(const void* vtx, const void* triIdx, uint32_t n, float* tri9, cudaStream_t st,
                                  std::string* err);

// Thread-local last error message (cl_last_error).
void setLastError(const std::string& msg);

// Process-wide: set once a tensor-core kernel reported that its bounded
// mbarrier wait ran out.  Its tensor memory may then have been released under
// a matrix operation still in flight, so the context is suspect and every
// later call that would launch a network kernel is refused (CL_ERR_STATE).
bool tcSuspect();
void markTcSuspect();
cl_status refuseIfTcSuspect(std::string* err);

} // namespace clb
