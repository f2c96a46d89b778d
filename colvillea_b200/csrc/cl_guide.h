// Hash-grid + tensor-core MLP networks, host side: parameters, Adam state and
// the kernels' launch sequence.  Two instances: the
// guiding network and the radiance cache (no counterpart in the reference
// renderer).
#pragma once

#include "cl_guide.cuh"
#include "cl_internal.h"

#include <type_traits>

namespace clb
{
// One training record in device memory (4 float4):
// {p.xyz in [0,1]^3, w} {n.xyz, -} {wo.xyz, -} {y.xyz, yw}, where y, yw are
// the guide's sampled direction and its BSDF pdf, or the cache's target RGB.
constexpr int kRecordF4 = 4;

struct GuideLoss; // -log p of the vMF mixture (or of the one-sample MIS density)
struct CacheLoss; // relative L2 of the predicted radiance

template <class S, class L> class HashNet
{
public:
    // Host record floats: guide {in9, omega, w, BSDF pdf}, cache {in9, RGB}.
    static constexpr int kRecFloats = std::is_same<S, guide::GuideShape>::value ? 14 : 12;

    explicit HashNet(const cl_guide_config& c);
    ~HashNet();
    cl_status init(cudaStream_t st, std::string* err);

    uint64_t paramCount() const { return hashParams_ + uint64_t(S::kParams); }
    uint64_t hashParams() const { return hashParams_; }
    const cl_guide_config& config() const { return cfg_; }
    const uint32_t* resolutions() const { return res_; }

    cl_status setParams(const float* p, uint64_t n, std::string* err);
    cl_status getParams(float* p, uint64_t n, std::string* err);
    cl_status forward(const float* in9, uint32_t n, float* out, std::string* err);
    cl_status gradient(const float* rec, uint32_t n, double* loss, float* grad, std::string* err);
    cl_status trainStepHost(const float* rec, uint32_t n, double* loss, std::string* err);
    cl_status sample(const float* in9, const float* u3, uint32_t n, float* dir, float* pdf, std::string* err);
    cl_status pdf(const float* in9, const float* dir, uint32_t n, float* pdf, std::string* err);

    // Device-side use: one training step on the records rec[0, min(*count,
    // batch)) (count in device memory), enqueued on the network's stream.
    // The loss lands in lossDev (device double) when the stream reaches it.
    cl_status trainDevice(const float4* rec, const uint32_t* count, std::string* err);
    guide::GridView grid() const;
    const uint4*    tcWeights() const { return wt_.as<uint4>(); }
    const double*   lossDev() const { return scal_.as<double>() + 1; }
    // Device error flags of the last training step (kTcTimeout), read with its loss.
    uint32_t*       trainErr() const { return reinterpret_cast<uint32_t*>(scal_.as<unsigned char>() + 52); }
    cl_status       checkTrainErr(std::string* err);
    uint64_t        steps() const { return step_; }

private:
    cl_status upload(const float* rec, uint32_t n, std::string* err);
    cl_status computeGradient(const float4* rec, const uint32_t* count, std::string* err);
    cl_status refreshCopies(std::string* err);

    cl_guide_config cfg_;
    uint32_t        res_[guide::kLevels] = {};
    uint32_t        denseMask_ = 0;
    uint64_t        hashParams_ = 0;
    cudaStream_t    st_ = nullptr;
    int             numSMs_ = 148;
    uint64_t        step_ = 0;

    DevBuf params_, grad_, m_, v_; // FP32 [hash | mlp]
    DevBuf table_;                 // bf16 copy of the hash table
    DevBuf wt_;                    // bf16 weights in the tensor-core canonical layout
    DevBuf scal_;                  // {sum w, loss, count (u32), sum of clamped w}; byte 48: inference error
                                   // flags; byte 52: training error flags
    DevBuf rec_, io_, io2_;        // host-entry staging
    DevBuf enc_, aux_;             // training: encoded batch in tensor-core tiles, per-sample loss inputs
};

using GuideNet = HashNet<guide::GuideShape, GuideLoss>;
using CacheNet = HashNet<guide::CacheShape, CacheLoss>;

void guideDefaultConfig(cl_guide_config* c);
cl_status guideResolutions(float nmin, float nmax, uint32_t* res);

} // namespace clb
