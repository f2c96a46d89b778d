// Hash-grid + tensor-core MLP networks of the path tracer (no counterpart in
// the reference renderer): the guiding network and the radiance cache share
// the encoding, the fused training forward/backward pass, the
// weight-gradient reduction over the batch and Adam; they differ in shape
// (MlpShape) and in the loss at the head (GuideLoss, CacheLoss).
#include "cl_guide.h"
#include "cl_mlp_tc.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <type_traits>
#include <vector>

namespace clb
{
using namespace guide;

namespace
{
__device__ __forceinline__ uint32_t laneIdx() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    // splitmix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float uniformPM1(uint64_t seed, uint64_t i)
{
    uint64_t h = mix64(seed * 0x9e3779b97f4a7c15ull + i + 1);
    return float(int64_t(h >> 40) - (int64_t(1) << 23)) * (1.0f / float(1 << 23)); // [-1, 1)
}

// Hash entries U[-1e-4, 1e-4]; W_l Glorot-uniform sqrt(6 / (in + out)).
template <class S> __global__ void kInitParams(float* p, uint64_t hashN, uint32_t seed)
{
    uint64_t n = hashN + S::kParams;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    {
        float u = uniformPM1(seed, i);
        if (i < hashN)
            p[i] = 1e-4f * u;
        else
        {
            int o = int(i - hashN), l = 0;
            while (l < S::kLayers - 1 && o >= S::woff(l + 1)) ++l;
            p[i] = u * sqrtf(6.0f / float(S::in(l) + S::out(l)));
        }
    }
}

__global__ void kTableCopy(const float* __restrict__ p, __nv_bfloat16* __restrict__ t, uint64_t n)
{
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        t[i] = __float2bfloat16_rn(p[i]);
}

// The weights as bf16 in the tensor-core canonical layout (cl_mlp_tc.cuh):
// 16-byte chunk e of layer l, at byte 2 woff(l) + 16 e, holds
// W[e % N][8 (e / N) .. + 7] (N = the layer's outputs).
template <class S> __global__ void kFrags(const float* __restrict__ mlp, uint4* __restrict__ wt)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= S::kParams / 8) return;
    int l = 0;
    while (l < S::kLayers - 1 && e >= S::woff(l + 1) / 8) ++l;
    const int    loc = e - S::woff(l) / 8, N = S::out(l), K = S::in(l);
    const float* W   = mlp + S::woff(l) + (loc % N) * K + 8 * (loc / N);
    wt[e] = make_uint4(packBf16(W[0], W[1]), packBf16(W[2], W[3]), packBf16(W[4], W[5]), packBf16(W[6], W[7]));
}
template <class S> constexpr int fragThreads() { return S::kParams / 8; }

__device__ __forceinline__ f3 ldf3(const float* p) { return {p[0], p[1], p[2]}; }

// Forward pass of `n` host-given samples (in9 rows) -> raw outputs, on the
// tensor-core path of the integrator's inference (cl_mlp_tc.cuh): 128-row
// tiles, thread t encodes row t and receives its outputs.
template <class S>
__global__ void __launch_bounds__(kTcThreads) kInferUnit(GridView g, const uint4* __restrict__ wt,
                                                         const float* __restrict__ in9, uint32_t n,
                                                         float* __restrict__ out, uint32_t* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t tmem  = tcSetup<S>(smem, wt);
    uint32_t       phase = 0u;
    for (uint32_t base = blockIdx.x * kTcRows; base < n; base += gridDim.x * kTcRows)
    {
        const uint32_t i = base + threadIdx.x;
        __align__(16) __nv_bfloat16 row[kIn];
        if (i < n)
        {
            const float* r = in9 + 9 * size_t(i);
            encodeRow(g, ldf3(r), ldf3(r + 3), ldf3(r + 6), row);
        }
        else
            zeroRow(row);
        uint32_t packed[kIn / 2];
#pragma unroll
        for (int q = 0; q < kIn / 2; ++q) packed[q] = reinterpret_cast<const uint32_t*>(row)[q];
        float o[S::kOut];
        if (!tcForward<S>(smem, tmem, packed, phase, o))
        {
            if (threadIdx.x == 0) atomicOr(err, kTcTimeout);
            break;
        }
        if (i < n)
            for (int c = 0; c < S::kOut; ++c) out[size_t(i) * S::kOut + c] = o[c];
    }
    tcTeardown(tmem);
}

// Mixture sample / pdf of given guide outputs (the network's mixture alone).
__global__ void kSampleUnit(const float* __restrict__ out48, const float* __restrict__ u3, uint32_t n,
                            float* __restrict__ dir, float* __restrict__ pdf)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Lobes L;
    headLobes(out48 + size_t(i) * kOut, &L);
    f3 d         = mixtureSample(L, u3[3 * i], u3[3 * i + 1], u3[3 * i + 2]);
    dir[3 * i]     = d.x;
    dir[3 * i + 1] = d.y;
    dir[3 * i + 2] = d.z;
    pdf[i]         = mixturePdf(L, d);
}
__global__ void kPdfUnit(const float* __restrict__ out48, const float* __restrict__ dir, uint32_t n,
                         float* __restrict__ pdf)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Lobes L;
    headLobes(out48 + size_t(i) * kOut, &L);
    pdf[i] = mixturePdf(L, f3{dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]});
}

// ---------------------------------------------------------------------------
// Training
// ---------------------------------------------------------------------------
struct TrainArgs
{
    const float4* __restrict__ rec;
    const uint32_t* count;
    uint32_t        batch;
    GridView        g;
    const uint4* __restrict__ wt; // canonical bf16 weights (tensor-core layout)
    float2*        gradTable;
    float*         gradMlp;       // FP32 weight gradients (the parameters after the hash table)
    uint32_t*      err;           // device error flags (kTcTimeout)
    double*        scal;     // [0] sum of weights, [1] loss, [3] sum of clamped weights
    int            learnSel; // guide: learned selection probability
    float          clamp;    // weight clamp (x batch mean), 0 = off
    uint4*         enc;      // encoded inputs: per 128-sample tile, 24,576 B in the tensor-core tile layout
    float4*        aux;      // per sample: {p.xyz (clamped to the unit cube), training weight / sum}, then the
                             // record's 4th float4 (guide: omega, BSDF pdf; cache: target RGB)
};

// Training weight of a record: clamped to clamp x the batch mean when set.
__device__ __forceinline__ float trainWeight(float w, const TrainArgs& a, uint32_t nB)
{
    if (a.clamp > 0.0f && nB > 0u) w = fminf(w, a.clamp * float(a.scal[0] / double(nB)));
    return w;
}

// A step trains on B = min(count, batch) samples; when more records were
// collected, sample j takes record floor(j * count / B) (an even subsample).
__device__ __forceinline__ uint32_t recordOf(uint32_t j, uint32_t count, uint32_t nB)
{
    return count > nB ? uint32_t(uint64_t(j) * count / nB) : j;
}

// Sum of the batch's weights into scal[slot] (slot 0: raw; slot 3: clamped,
// after slot 0 is complete).
__global__ void kTrainPrep(TrainArgs a, int slot)
{
    __shared__ double part[32];
    const uint32_t count = *a.count, nB = min(count, a.batch);
    double         s     = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nB; j += gridDim.x * blockDim.x)
    {
        float w = a.rec[kRecordF4 * size_t(recordOf(j, count, nB))].w;
        s += double(slot ? trainWeight(w, a, nB) : w);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (laneIdx() == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += part[w];
        if (t != 0.0) atomicAdd(&a.scal[slot], t);
    }
}

// log p(omega) of the mixture given by the head outputs o[0..47], and its
// gradient with respect to o (grad[40..47] = 0: unused outputs).
__device__ __forceinline__ float headLossGrad(const float* o, f3 om, float* grad)
{
    float mx = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
    float e[kLobes], S = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        e[k] = expf(o[5 * k + 4] - mx);
        S += e[k];
    }
    const float logS = logf(S);
    float       lp[kLobes], kap[kLobes], c[kLobes], nrm[kLobes];
    f3          mu[kLobes];
    float       m = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        f3 raw{o[5 * k], o[5 * k + 1], o[5 * k + 2]};
        nrm[k]   = fmaxf(sqrtf(dot(raw, raw)), 1e-6f);
        mu[k]    = raw * (1.0f / nrm[k]);
        float lk = fminf(fmaxf(o[5 * k + 3], kKappaMin), kKappaMax);
        kap[k]   = expf(lk);
        c[k]     = dot(mu[k], om);
        lp[k]    = (o[5 * k + 4] - mx - logS) + lk - logf(2.0f * kPiF) - logf(-expm1f(-2.0f * kap[k])) +
                kap[k] * (c[k] - 1.0f);
        m = fmaxf(m, lp[k]);
    }
    float R = 0.0f, r[kLobes];
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        r[k] = expf(lp[k] - m);
        R += r[k];
    }
    const float invR = 1.0f / R;
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        float rk       = r[k] * invR;
        grad[5 * k + 4] = rk - e[k] / S;
        float lkr      = o[5 * k + 3];
        float dlk      = 1.0f / kap[k] - 2.0f * expf(-2.0f * kap[k]) / -expm1f(-2.0f * kap[k]) + (c[k] - 1.0f);
        grad[5 * k + 3] = (lkr > kKappaMin && lkr < kKappaMax) ? rk * dlk * kap[k] : 0.0f;
        f3    dm       = om * kap[k];
        float pr       = dot(dm, mu[k]);
        f3    proj     = dm - mu[k] * pr;
        float sc       = rk / nrm[k];
        grad[5 * k]     = proj.x * sc;
        grad[5 * k + 1] = proj.y * sc;
        grad[5 * k + 2] = proj.z * sc;
    }
#pragma unroll
    for (int k = 5 * kLobes; k < kOut; ++k) grad[k] = 0.0f;
    return m + logf(R);
}

} // namespace

// Per-sample loss l(o) and dl/do of the guiding network: -log p_guide(omega),
// or with the learned selection probability -log((1 - a) p_bsdf + a p_guide)
// (lobe gradients scaled by a p_guide / p_mix, selection logit
// (p_guide - p_bsdf) / p_mix da/dlogit).  Record: omega in r3.xyz, the BSDF
// pdf of omega in r3.w.
struct GuideLoss
{
    static constexpr int kOut = GuideShape::kOut;
    __device__ static float eval(const float* o, float4 r3, int learnSel, float* grad)
    {
        float lp = headLossGrad(o, f3{r3.x, r3.y, r3.z}, grad);
        if (learnSel)
        {
            const float x  = o[kSelOut];
            const float sg = 1.0f / (1.0f + expf(-x));
            const float al = kSelMin + (kSelMax - kSelMin) * sg;
            const float pg = expf(lp), pb = r3.w;
            const float pm = fmaxf((1.0f - al) * pb + al * pg, 1e-30f);
            const float sc = al * pg / pm;
#pragma unroll
            for (int c = 0; c < 5 * kLobes; ++c) grad[c] *= sc;
            grad[kSelOut] = (pg - pb) / pm * (kSelMax - kSelMin) * sg * (1.0f - sg);
            lp            = logf(pm);
        }
#pragma unroll
        for (int c = 0; c < kOut; ++c) grad[c] = -grad[c];
        return -lp;
    }
};

// Radiance cache: relative L2 of the RGB prediction o[0..2] against the
// path-traced target r3.xyz (Mueller et al. 2021): mean over the channels of
// (o - y)^2 / (o^2 + 0.01), the denominator held constant in the gradient.
struct CacheLoss
{
    static constexpr int kOut = CacheShape::kOut;
    __device__ static float eval(const float* o, float4 r3, int, float* grad)
    {
        const float y[3] = {r3.x, r3.y, r3.z};
        float       l    = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
            const float d = o[c] - y[c], den = o[c] * o[c] + 0.01f;
            l += d * d / den;
            grad[c] = (2.0f / 3.0f) * d / den;
        }
#pragma unroll
        for (int c = 3; c < kOut; ++c) grad[c] = 0.0f;
        return l * (1.0f / 3.0f);
    }
};

namespace
{
// ---------------------------------------------------------------------------
// Training on the fifth-generation tensor cores (tcgen05): one kernel per
// step does, for each 128-sample tile of the batch, the encoding, the
// forward pass, the loss at the head, the backward pass and the weight
// gradients.  A CTA of 128 threads owns one tile at a time, thread t sample
// t (its hash-grid position stays in registers):
//   forward, layer l:  acc[128 x out] = a_l[128 x in] . W_l^T   (M = 128,
//                      A and B K-major) -> ReLU -> bf16 -> a_{l+1} (smem);
//   head:              dl/do x (w / sum w) -> bf16 -> delta (smem);
//   backward, layer l: dW_l[out x in] += delta^T . a_l  (M = 64, both
//                      operands MN-major views of the same smem tiles, K =
//                      the 128 samples; accumulated in TMEM over all of the
//                      CTA's tiles), and acc[128 x in] = delta . W_l
//                      (B = the MN-major view of the forward weights),
//                      masked by ReLU'(a_l) -> bf16 -> delta of layer l-1;
//                      at layer 0 the product over the 32 hash-feature
//                      inputs is scattered to the hash table's gradient.
// Every layer input of the tile stays in shared memory for the backward
// pass; nothing is staged through global memory.  At the end each CTA adds
// its weight gradients (TMEM, M = 64 layout: row r in lane 32 (r / 16) +
// r % 16) to the global gradient.
// ---------------------------------------------------------------------------
template <class S> struct TrainTc
{
    static constexpr int L  = S::kLayers - 1; // the output layer
    static constexpr int kW = S::kParams * 2; // canonical bf16 weights (cl_mlp_tc.cuh)
    static constexpr int kA0 = kTcRows * kIn * 2;  // an encoded-input tile (24,576 B)
    // Input tile of layer l (128 rows, canonical K-major, 2048 B per 8-column chunk); layer 0's input is one of
    // two encoded-tile buffers (a0(b)): the next tile's bulk copy fills the other one.
    __host__ __device__ static constexpr int a0(int b) { return kW + b * kA0; }
    __host__ __device__ static constexpr int act(int l) { return kW + 2 * kA0 + (l - 1) * kTcRows * kWidth * 2; }
    static constexpr int kDelta = act(S::kLayers); // output-gradient tile, 64 columns (zero-padded)
    static constexpr int kBar   = kDelta + kTcRows * kWidth * 2; // MMA mbarrier, TMEM address, 2 load mbarriers
    static constexpr int kSmem  = kBar + 32;
    // TMEM: columns [0, 64) the layer accumulator; then dW_l (M = 64) at dw(l).
    __host__ __device__ static constexpr uint32_t dw(int l) { return 64u + (l == 0 ? 0u : uint32_t(kIn + (l - 1) * kWidth)); }
    static constexpr uint32_t kCols = 512;
    static_assert(kW % 16 == 0, "weights: 16-byte chunks");
    static_assert(dw(S::kLayers) <= kCols, "weight gradients exceed tensor memory");
    static_assert(S::kOut <= kWidth, "output gradient tile is 64 columns wide");
};

__device__ __forceinline__ void tcSyncForMma()
{
    asyncProxyFence();
    tcFenceBefore();
    __syncthreads();
}

// Waits for the committed MMAs; false in every thread when the wait ran out.
__device__ __forceinline__ bool tcWaitAll(uint32_t bar, uint32_t& phase)
{
    const bool ok = mbarWait(bar, phase);
    phase ^= 1u;
    tcFenceAfter();
    return __syncthreads_and(ok) != 0;
}

// Encoding of the training batch, one thread per sample (many warps hide the
// hash-grid gathers): the 96 encoded inputs go to tile j / 128 in the
// tensor-core tile layout (chunk c of row r at c * 2048 + r * 16, so that a
// tile is one contiguous 24,576-byte block for the training kernel's bulk
// copy), with the sample's clamped position, normalised training weight and
// loss inputs beside it.  Rows past the batch in the last tile are zero.
__global__ void __launch_bounds__(256, 4) kTrainEncode(TrainArgs a)
{
    const uint32_t count = *a.count, nB = min(count, a.batch);
    const uint32_t rows  = (nB + kTcRows - 1) / kTcRows * kTcRows;
    const double   wsum  = a.clamp > 0.0f ? a.scal[3] : a.scal[0];
    const float    invW  = wsum > 0.0 ? float(1.0 / wsum) : 0.0f;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < rows; j += gridDim.x * blockDim.x)
    {
        uint32_t r[kIn / 2];
        float4   pw{0.0f, 0.0f, 0.0f, 0.0f}, r3{0.0f, 0.0f, 0.0f, 0.0f};
        if (j < nB)
        {
            const float4* R  = a.rec + kRecordF4 * size_t(recordOf(j, count, nB));
            const float4  r0 = R[0], r1 = R[1], r2 = R[2];
            r3               = R[3];
            const f3 p       = clampUnit(f3{r0.x, r0.y, r0.z});
            pw               = make_float4(p.x, p.y, p.z, trainWeight(r0.w, a, nB) * invW);
#pragma unroll
            for (int l = 0; l < kLevels; ++l)
            {
                const float2 f = encodeLevel(a.g, l, p);
                r[l]           = packBf16(f.x, f.y);
            }
            oneBlobPacked(f3{r1.x, r1.y, r1.z}, r + kHashF / 2);
            oneBlobPacked(f3{r2.x, r2.y, r2.z}, r + (kHashF + 2 * kBlob) / 2);
        }
        else
#pragma unroll
            for (int q = 0; q < kIn / 2; ++q) r[q] = 0u;
        uint4* tile = a.enc + size_t(j / kTcRows) * (kTcRows * kIn / 8);
#pragma unroll
        for (int c = 0; c < kIn / 8; ++c)
            tile[c * kTcRows + (j % kTcRows)] = make_uint4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
        a.aux[2 * size_t(j)]     = pw;
        a.aux[2 * size_t(j) + 1] = r3;
    }
}

// Two threads per sample row (256 per CTA): thread t serves row t % 128;
// half h = t / 128 encodes hash levels 8h .. 8h+7 and one of the two one-blob
// directions, converts columns 32h .. 32h+31 of each layer's accumulator
// (warps w and w + 4 read the same TMEM lanes), and scatters the hash-feature
// gradient of its 8 levels; the head's loss runs in half 0.
constexpr int kTrainThreads = 2 * kTcThreads;

template <class S, class LOSS> __global__ void __launch_bounds__(kTrainThreads, 1) kTrainTc(TrainArgs a)
{
    using T              = TrainTc<S>;
    constexpr int L      = T::L;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t count = *a.count, nB = min(count, a.batch);
    const uint32_t tiles = (nB + kTcRows - 1) / kTcRows;
    if (blockIdx.x >= tiles) return; // before any TMEM allocation
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u, row = t & (kTcRows - 1u), half = t >> 7;
    {
        uint4* w = reinterpret_cast<uint4*>(smem);
        for (int i = int(t); i < T::kW / 16; i += kTrainThreads) w[i] = __ldg(a.wt + i);
    }
    const uint32_t bar = smemAddr(smem + T::kBar);
    const uint32_t lbar[2] = {bar + 16u, bar + 24u}; // encoded-tile bulk copies into a0(0), a0(1)
    if (t == 0)
    {
        mbarInit(bar, 1u);
        mbarInit(lbar[0], 1u);
        mbarInit(lbar[1], 1u);
    }
    if (warp == 0) tmemAlloc(bar + 8u, T::kCols);
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem  = *reinterpret_cast<volatile uint32_t*>(smem + T::kBar + 8);
    const uint32_t tRow  = tmem + (((warp & 3u) * 32u) << 16); // this warp's TMEM lanes
    const uint32_t wS    = smemAddr(smem), dS = smemAddr(smem + T::kDelta);
    constexpr uint32_t kTileU4 = kTcRows * kIn / 8;
    if (t == 0) bulkLoad(smemAddr(smem + T::a0(0)), a.enc + size_t(blockIdx.x) * kTileU4, T::kA0, lbar[0]);
    uint32_t       phase = 0u, lphase[2] = {0u, 0u};
    int            pending = 1; // 1 + the buffer whose bulk copy was issued and not yet waited for (0: none)
    bool           first = true, ok = true;
    float          lossPart = 0.0f;
    uint32_t       it = 0u;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++it)
    {
        const uint32_t b     = it & 1u;
        const uint32_t j     = tile * kTcRows + row;
        const bool     valid = j < nB;
        const float4   pw    = a.aux[2 * size_t(j)];
        const float4   r3    = half == 0u ? a.aux[2 * size_t(j) + 1] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const f3       p{pw.x, pw.y, pw.z};
        const float    sw = pw.w;
        // This tile's encoded inputs (bulk copy issued one tile ahead), then the next tile's copy into
        // the other buffer, whose last readers (this CTA's previous MMAs) have completed.
        if (!__syncthreads_and(mbarWait(lbar[b], lphase[b])))
        {
            ok = false; // the copy may still land: `pending` keeps its buffer for the final wait
            break;
        }
        lphase[b] ^= 1u;
        pending = 0;
        if (tile + gridDim.x < tiles)
        {
            if (t == 0)
                bulkLoad(smemAddr(smem + T::a0(b ^ 1u)), a.enc + size_t(tile + gridDim.x) * kTileU4, T::kA0,
                         lbar[b ^ 1u]);
            pending = int(b ^ 1u) + 1;
        }
        // Forward.
        float o[S::kOut];
#pragma unroll 1
        for (int l = 0; l <= L && ok; ++l)
        {
            tcSyncForMma();
            if (t == 0)
            {
                tcFenceAfter();
                const int      K = S::in(l), N = S::out(l);
                const uint32_t aS = smemAddr(smem + (l == 0 ? T::a0(int(b)) : T::act(l)));
                const uint32_t wl = wS + 2u * uint32_t(S::woff(l));
                for (int ks = 0; ks < K / 16; ++ks)
                    tcMma(tmem, tcDesc(aS + uint32_t(ks) * 2u * kTcChunk, kTcChunk, 128u),
                          tcDesc(wl + uint32_t(ks * 2 * N * 16), uint32_t(N * 16), 128u), tcIdescMaj(128, N, false, false),
                          ks > 0 ? 1u : 0u);
                tcCommit(bar);
            }
            ok = tcWaitAll(bar, phase);
            if (!ok) break;
            if (l < L)
            {
                uint32_t v[2][16];
#pragma unroll
                for (int c = 0; c < 2; ++c) tmemLd16(tRow + 32u * half + uint32_t(16 * c), v[c]);
                tmemWait();
                unsigned char* nxt = smem + T::act(l + 1);
#pragma unroll
                for (int c = 0; c < 2; ++c)
                {
                    *tileChunk(nxt, row, int(4 * half) + 2 * c)     = packRelu8(v[c]);
                    *tileChunk(nxt, row, int(4 * half) + 2 * c + 1) = packRelu8(v[c] + 8);
                }
            }
            else
            {
                uint32_t v[S::kOut / 16][16];
#pragma unroll
                for (int c = 0; c < S::kOut / 16; ++c) tmemLd16(tRow + uint32_t(16 * c), v[c]);
                tmemWait();
#pragma unroll
                for (int c = 0; c < S::kOut / 16; ++c)
#pragma unroll
                    for (int q = 0; q < 16; ++q) o[16 * c + q] = __uint_as_float(v[c][q]);
            }
        }
        if (!ok) break;
        // Loss and output gradient (half 0) -> delta row (columns >= kOut zero).
        if (half == 0u)
        {
            float gr[S::kOut];
            if (valid)
            {
                lossPart += sw * LOSS::eval(o, r3, a.learnSel, gr);
#pragma unroll
                for (int c = 0; c < S::kOut; ++c) gr[c] *= sw;
            }
            else
#pragma unroll
                for (int c = 0; c < S::kOut; ++c) gr[c] = 0.0f;
            unsigned char* d = smem + T::kDelta;
#pragma unroll
            for (int c = 0; c < kWidth / 8; ++c)
            {
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (8 * c < S::kOut)
                    v = make_uint4(packBf16(gr[8 * c], gr[8 * c + 1]), packBf16(gr[8 * c + 2], gr[8 * c + 3]),
                                   packBf16(gr[8 * c + 4], gr[8 * c + 5]), packBf16(gr[8 * c + 6], gr[8 * c + 7]));
                *tileChunk(d, row, c) = v;
            }
        }
        // Backward.
#pragma unroll 1
        for (int l = L; l >= 0 && ok; --l)
        {
            tcSyncForMma();
            if (t == 0)
            {
                tcFenceAfter();
                const int      K = S::out(l), I = S::in(l), N = l > 0 ? I : kHashF;
                const uint32_t aS = smemAddr(smem + (l == 0 ? T::a0(int(b)) : T::act(l)));
                const uint32_t wl = wS + 2u * uint32_t(S::woff(l));
                // dW_l += delta^T a_l: A = delta (M = 64 output units, MN-major), B = a_l (N = I inputs,
                // MN-major), K = 16 samples per instruction.
                for (int ks = 0; ks < kTcRows / 16; ++ks)
                    tcMma(tmem + T::dw(l), tcDesc(dS + uint32_t(ks) * 256u, 128u, kTcChunk),
                          tcDesc(aS + uint32_t(ks) * 256u, 128u, kTcChunk), tcIdescMaj(64, I, true, true),
                          (first && ks == 0) ? 0u : 1u);
                // acc = delta . W_l: A = delta (K-major, K = the layer's outputs), B = W_l viewed with
                // N = its inputs (MN-major: 8-input groups 16 K bytes apart, 8-output groups 128 B).
                for (int ks = 0; ks < K / 16; ++ks)
                    tcMma(tmem, tcDesc(dS + uint32_t(ks) * 2u * kTcChunk, kTcChunk, 128u),
                          tcDesc(wl + uint32_t(ks) * 256u, 128u, uint32_t(16 * K)), tcIdescMaj(128, N, false, true),
                          ks > 0 ? 1u : 0u);
                tcCommit(bar);
            }
            ok = tcWaitAll(bar, phase);
            if (!ok) break;
            if (l > 0)
            {
                // delta of layer l-1 = acc masked by ReLU'(a_l) (a zero bf16 input was a unit that was off);
                // this half's 32 columns.
                uint32_t v[2][16];
#pragma unroll
                for (int c = 0; c < 2; ++c) tmemLd16(tRow + 32u * half + uint32_t(16 * c), v[c]);
                tmemWait();
                const unsigned char* al = smem + T::act(l);
                unsigned char*       d  = smem + T::kDelta;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    const int       cc    = int(4 * half) + c;
                    const uint4     m     = *tileChunk(const_cast<unsigned char*>(al), row, cc);
                    const uint32_t  mw[4] = {m.x, m.y, m.z, m.w};
                    const uint32_t* src   = v[c >> 1] + 8 * (c & 1);
                    uint32_t        pk[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                    {
                        const float lo = (mw[q] & 0xffffu) ? __uint_as_float(src[2 * q]) : 0.0f;
                        const float hi = (mw[q] >> 16) ? __uint_as_float(src[2 * q + 1]) : 0.0f;
                        pk[q]          = packBf16(lo, hi);
                    }
                    *tileChunk(d, row, cc) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
            }
            else
            {
                // Gradient of this half's 8 hash levels (FP32 columns 16h .. 16h+15: feature f of level l
                // is column 2 l + f).  The TMEM load is warp-collective: every lane takes part.
                uint32_t v[16];
                tmemLd16(tRow + 16u * half, v);
                tmemWait();
#pragma unroll
                for (int q = 0; q < 8; ++q)
                {
                    const float d0 = __uint_as_float(v[2 * q]), d1 = __uint_as_float(v[2 * q + 1]);
                    if (!valid || (d0 == 0.0f && d1 == 0.0f)) continue;
                    const int  lv = int(8 * half) + q;
                    const Cell c  = gridCell(a.g.res[lv], p);
                    float2*    gb = a.gradTable + (size_t(lv) << a.g.log2T);
                    uint32_t   idx[8];
                    float      w[8];
                    cornerIndices(a.g, lv, c, idx);
                    cornerWeights(c, w);
#pragma unroll
                    for (int k = 0; k < 8; ++k) atomicAdd(gb + idx[k], make_float2(w[k] * d0, w[k] * d1));
                }
            }
        }
        first = false;
    }
    // A bulk copy issued for a tile this CTA no longer processes (a wait ran out) must land before the
    // CTA's shared memory is released: wait for it, again with a bound.
    if (pending) mbarWait(lbar[pending - 1], lphase[pending - 1]);
    for (int off = 16; off > 0; off >>= 1) lossPart += __shfl_xor_sync(0xffffffffu, lossPart, off);
    if (lane == 0 && lossPart != 0.0f) atomicAdd(&a.scal[1], double(lossPart));
    if (!ok)
    {
        if (t == 0) atomicOr(a.err, kTcTimeout);
    }
    else if (!first)
    {
        // Weight gradients: row r of dW_l (M = 64) is in TMEM lane 32 (r / 16) + r % 16, so warps w and
        // w + 4 hold rows 16 (w % 4) .. + 15 in their lanes 0-15; the halves take alternate 16-column groups.
        const int o = int(warp & 3u) * 16 + int(lane);
#pragma unroll 1
        for (int l = 0; l <= L; ++l)
        {
            const int I = S::in(l);
            float*    G = a.gradMlp + S::woff(l);
#pragma unroll 1
            for (int c = int(half); c < I / 16; c += 2)
            {
                uint32_t v[16];
                tmemLd16(tRow + T::dw(l) + uint32_t(16 * c), v);
                tmemWait();
                if (lane < 16u && o < S::out(l))
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                    {
                        const float x = __uint_as_float(v[q]);
                        if (x != 0.0f) atomicAdd(G + o * I + 16 * c + q, x);
                    }
            }
        }
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0) tmemFree(tmem, T::kCols);
}

// Adam (FP32 master parameters) over float4 groups - the hash block and
// every weight block hold multiples of 4 floats - with two groups in flight
// per thread; clears the gradient it consumed and refreshes the bf16 copy
// of the hash table.  a = lr / (1 - beta1^t), ic2 = 1 / (1 - beta2^t).
struct AdamK
{
    float b1, b2, eps, a, ic2;
};
__device__ __forceinline__ float adam1(float p, float& m, float& v, float g, const AdamK& k)
{
    m = k.b1 * m + (1.0f - k.b1) * g;
    v = k.b2 * v + (1.0f - k.b2) * g * g;
    return p - __fdividef(k.a * m, sqrtf(v * k.ic2) + k.eps);
}
__device__ __forceinline__ void adam4(float4* __restrict__ p, float4* __restrict__ grad, float4* __restrict__ m,
                                      float4* __restrict__ v, uint2* __restrict__ table, uint64_t i, uint64_t hash4,
                                      float4 g, float4 mi, float4 vi, float4 pi, const AdamK& k)
{
    pi.x = adam1(pi.x, mi.x, vi.x, g.x, k);
    pi.y = adam1(pi.y, mi.y, vi.y, g.y, k);
    pi.z = adam1(pi.z, mi.z, vi.z, g.z, k);
    pi.w = adam1(pi.w, mi.w, vi.w, g.w, k);
    grad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    m[i]    = mi;
    v[i]    = vi;
    p[i]    = pi;
    if (i < hash4) table[i] = make_uint2(packBf16(pi.x, pi.y), packBf16(pi.z, pi.w));
}
__global__ void __launch_bounds__(256) kAdam(float4* __restrict__ p, float4* __restrict__ grad,
                                             float4* __restrict__ m, float4* __restrict__ v, uint64_t n4,
                                             uint64_t hash4, AdamK k, uint2* __restrict__ table)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint64_t       i      = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    for (; i + stride < n4; i += 2 * stride)
    {
        const uint64_t j  = i + stride;
        float4         g0 = grad[i], m0 = m[i], v0 = v[i], p0 = p[i];
        float4         g1 = grad[j], m1 = m[j], v1 = v[j], p1 = p[j];
        adam4(p, grad, m, v, table, i, hash4, g0, m0, v0, p0, k);
        adam4(p, grad, m, v, table, j, hash4, g1, m1, v1, p1, k);
    }
    if (i < n4) adam4(p, grad, m, v, table, i, hash4, grad[i], m[i], v[i], p[i], k);
}

int gridFor(uint64_t n, int block, int cap)
{
    uint64_t b = (n + block - 1) / block;
    return int(b < uint64_t(cap) ? (b ? b : 1) : cap);
}

} // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
void guideDefaultConfig(cl_guide_config* c)
{
    std::memset(c, 0, sizeof(*c));
    c->log2_table      = 19;
    c->n_min           = 16.0f;
    c->n_max           = 1024.0f;
    c->learning_rate   = 1e-2f;
    c->beta1           = 0.9f;
    c->beta2           = 0.99f;
    c->epsilon         = 1e-10f;
    c->bsdf_fraction   = 0.5f;
    c->batch           = 1u << 18;
    c->train_spp       = 32;
    c->class_mask      = 7u;
    c->seed            = 1;
    c->learn_selection = 0u;
    c->weight_clamp    = 0.0f;
    c->min_depth       = 1u;
    c->min_alpha       = 0.0f;
}

cl_status guideResolutions(float nmin, float nmax, uint32_t* res)
{
    if (!(nmin >= 1.0f) || !(nmax >= nmin) || nmax > 16777216.0f) return CL_ERR_INVALID_ARG;
    double b = std::exp((std::log(double(nmax)) - std::log(double(nmin))) / double(kLevels - 1));
    for (int l = 0; l < kLevels; ++l) res[l] = uint32_t(std::floor(double(nmin) * std::pow(b, double(l))));
    return CL_OK;
}

template <class S, class L> HashNet<S, L>::HashNet(const cl_guide_config& c) : cfg_(c) {}
template <class S, class L> HashNet<S, L>::~HashNet() = default;

template <class S, class L> cl_status HashNet<S, L>::init(cudaStream_t st, std::string* err)
{
    st_ = st;
    if (cfg_.log2_table < 8 || cfg_.log2_table > 24)
    {
        *err = "network: log2_table must be in [8, 24]";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg_.batch == 0 || cfg_.batch > (1u << 24) || !(cfg_.learning_rate > 0.0f) || !(cfg_.bsdf_fraction >= 0.0f) ||
        !(cfg_.bsdf_fraction <= 1.0f) || !(cfg_.beta1 >= 0.0f && cfg_.beta1 < 1.0f) ||
        !(cfg_.beta2 >= 0.0f && cfg_.beta2 < 1.0f) || !(cfg_.epsilon >= 0.0f) || cfg_.learn_selection > 1u ||
        !(cfg_.weight_clamp >= 0.0f) || !(cfg_.min_alpha >= 0.0f && cfg_.min_alpha <= 1.0f))
    {
        *err = "network: batch, learning rate, Adam, bsdf_fraction, learn_selection, weight_clamp or min_alpha out of "
               "range";
        return CL_ERR_INVALID_ARG;
    }
    bool given = false;
    for (int l = 0; l < kLevels; ++l) given |= cfg_.resolutions[l] != 0u;
    if (given)
    {
        for (int l = 0; l < kLevels; ++l)
        {
            if (cfg_.resolutions[l] < 1u || cfg_.resolutions[l] > (1u << 24))
            {
                *err = "network: resolutions must be in [1, 2^24]";
                return CL_ERR_INVALID_ARG;
            }
            res_[l] = cfg_.resolutions[l];
        }
    }
    else if (guideResolutions(cfg_.n_min, cfg_.n_max, res_) != CL_OK)
    {
        *err = "network: n_min/n_max out of range";
        return CL_ERR_INVALID_ARG;
    }
    const uint64_t T = 1ull << cfg_.log2_table;
    denseMask_       = 0;
    for (int l = 0; l < kLevels; ++l)
    {
        uint64_t r1 = uint64_t(res_[l]) + 1;
        if (r1 * r1 * r1 <= T) denseMask_ |= 1u << l;
    }
    hashParams_ = uint64_t(kLevels) * T * kFeat;
    const uint64_t n = paramCount();
    int dev = 0;
    CL_CUDA(cudaGetDevice(&dev), err);
    CL_CUDA(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, dev), err);
    CL_CUDA(cudaFuncSetAttribute(kInferUnit<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<S>::kSmem),
            err);
    CL_CUDA(cudaFuncSetAttribute(kInferUnit<S>, cudaFuncAttributePreferredSharedMemoryCarveout, 100), err);
    CL_CUDA(cudaFuncSetAttribute(kTrainTc<S, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, TrainTc<S>::kSmem), err);
    CL_TRY(params_.alloc(n * 4, err));
    CL_TRY(grad_.alloc(n * 4, err));
    CL_TRY(m_.alloc(n * 4, err));
    CL_TRY(v_.alloc(n * 4, err));
    CL_TRY(table_.alloc(hashParams_ * 2, err));
    CL_TRY(wt_.alloc(TcLayout<S>::kWBytes, err));
    CL_TRY(scal_.alloc(64, err));
    {
        const size_t tiles = (size_t(cfg_.batch) + kTcRows - 1) / kTcRows;
        CL_TRY(enc_.alloc(tiles * TrainTc<S>::kA0, err));
        CL_TRY(aux_.alloc(tiles * kTcRows * 32, err));
    }
    kInitParams<S><<<gridFor(n, 256, numSMs_ * 8), 256, 0, st_>>>(params_.f(), hashParams_, cfg_.seed);
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemsetAsync(grad_.p, 0, n * 4, st_), err);
    CL_CUDA(cudaMemsetAsync(m_.p, 0, n * 4, st_), err);
    CL_CUDA(cudaMemsetAsync(v_.p, 0, n * 4, st_), err);
    CL_CUDA(cudaMemsetAsync(scal_.p, 0, 64, st_), err);
    step_ = 0;
    CL_TRY(refreshCopies(err));
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

template <class S, class L> GridView HashNet<S, L>::grid() const
{
    GridView g;
    g.table     = table_.as<const __nv_bfloat162>();
    g.log2T     = cfg_.log2_table;
    g.mask      = (1u << cfg_.log2_table) - 1u;
    g.denseMask = denseMask_;
    for (int l = 0; l < kLevels; ++l) g.res[l] = res_[l];
    return g;
}

template <class S, class L> cl_status HashNet<S, L>::refreshCopies(std::string* err)
{
    kTableCopy<<<gridFor(hashParams_, 256, numSMs_ * 8), 256, 0, st_>>>(params_.f(), table_.as<__nv_bfloat16>(),
                                                                        hashParams_);
    CL_CUDA(cudaGetLastError(), err);
    kFrags<S><<<(fragThreads<S>() + 255) / 256, 256, 0, st_>>>(params_.f() + hashParams_, wt_.as<uint4>());
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

template <class S, class L> cl_status HashNet<S, L>::setParams(const float* p, uint64_t n, std::string* err)
{
    if (!p || n != paramCount())
    {
        *err = "network: parameter count mismatch";
        return CL_ERR_INVALID_ARG;
    }
    CL_CUDA(cudaMemcpyAsync(params_.p, p, n * 4, cudaMemcpyHostToDevice, st_), err);
    CL_CUDA(cudaMemsetAsync(grad_.p, 0, n * 4, st_), err);
    CL_CUDA(cudaMemsetAsync(m_.p, 0, n * 4, st_), err);
    CL_CUDA(cudaMemsetAsync(v_.p, 0, n * 4, st_), err);
    step_ = 0;
    CL_TRY(refreshCopies(err));
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

template <class S, class L> cl_status HashNet<S, L>::getParams(float* p, uint64_t n, std::string* err)
{
    if (!p || n != paramCount())
    {
        *err = "network: parameter count mismatch";
        return CL_ERR_INVALID_ARG;
    }
    CL_CUDA(cudaMemcpyAsync(p, params_.p, n * 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::forward(const float* in9, uint32_t n, float* out, std::string* err)
{
    if ((!in9 || !out) && n)
    {
        *err = "network: null buffer";
        return CL_ERR_INVALID_ARG;
    }
    if (n == 0) return CL_OK;
    CL_TRY(io_.alloc(size_t(n) * 9 * 4, err));
    CL_TRY(io2_.alloc(size_t(n) * S::kOut * 4, err));
    CL_CUDA(cudaMemcpyAsync(io_.p, in9, size_t(n) * 9 * 4, cudaMemcpyHostToDevice, st_), err);
    uint32_t* flag = reinterpret_cast<uint32_t*>(scal_.as<unsigned char>() + 48);
    CL_CUDA(cudaMemsetAsync(flag, 0, 4, st_), err);
    kInferUnit<S><<<gridFor(n, kTcRows, numSMs_ * 2), kTcThreads, TcLayout<S>::kSmem, st_>>>(grid(), tcWeights(),
                                                                                            io_.f(), n, io2_.f(), flag);
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemcpyAsync(out, io2_.p, size_t(n) * S::kOut * 4, cudaMemcpyDeviceToHost, st_), err);
    uint32_t hf = 0u;
    CL_CUDA(cudaMemcpyAsync(&hf, flag, 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    if (hf & kTcTimeout)
    {
        markTcSuspect();
        *err = "network: a tensor-core wait ran out";
        return CL_ERR_TIMEOUT;
    }
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::sample(const float* in9, const float* u3, uint32_t n, float* dir, float* pdf,
                                std::string* err)
{
    if (!std::is_same<S, GuideShape>::value)
    {
        *err = "sampling is defined for the guiding network only";
        return CL_ERR_STATE;
    }
    if (n == 0) return CL_OK;
    if (!in9 || !u3 || !dir || !pdf)
    {
        *err = "network: null buffer";
        return CL_ERR_INVALID_ARG;
    }
    std::vector<float> out(size_t(n) * S::kOut);
    CL_TRY(forward(in9, n, out.data(), err));
    DevBuf u, d, p;
    CL_TRY(u.alloc(size_t(n) * 12, err));
    CL_TRY(d.alloc(size_t(n) * 12, err));
    CL_TRY(p.alloc(size_t(n) * 4, err));
    CL_CUDA(cudaMemcpyAsync(u.p, u3, size_t(n) * 12, cudaMemcpyHostToDevice, st_), err);
    kSampleUnit<<<(n + 127) / 128, 128, 0, st_>>>(io2_.f(), u.f(), n, d.f(), p.f());
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemcpyAsync(dir, d.p, size_t(n) * 12, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaMemcpyAsync(pdf, p.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::pdf(const float* in9, const float* dir, uint32_t n, float* pdf, std::string* err)
{
    if (!std::is_same<S, GuideShape>::value)
    {
        *err = "the pdf is defined for the guiding network only";
        return CL_ERR_STATE;
    }
    if (n == 0) return CL_OK;
    if (!in9 || !dir || !pdf)
    {
        *err = "network: null buffer";
        return CL_ERR_INVALID_ARG;
    }
    std::vector<float> out(size_t(n) * S::kOut);
    CL_TRY(forward(in9, n, out.data(), err));
    DevBuf d, p;
    CL_TRY(d.alloc(size_t(n) * 12, err));
    CL_TRY(p.alloc(size_t(n) * 4, err));
    CL_CUDA(cudaMemcpyAsync(d.p, dir, size_t(n) * 12, cudaMemcpyHostToDevice, st_), err);
    kPdfUnit<<<(n + 127) / 128, 128, 0, st_>>>(io2_.f(), d.f(), n, p.f());
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemcpyAsync(pdf, p.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

// Host records (kRecFloats per row) -> device records; the record count
// goes to scal[2] (u32).  Guide rows: in9, omega, w, BSDF pdf of omega;
// cache rows: in9, target RGB (weight 1).
template <class S, class L> cl_status HashNet<S, L>::upload(const float* rec, uint32_t n, std::string* err)
{
    if (!rec || n == 0)
    {
        *err = "network: empty or null batch";
        return CL_ERR_INVALID_ARG;
    }
    constexpr int      kf = kRecFloats;
    std::vector<float> h(size_t(n) * 16, 0.0f);
    for (uint32_t i = 0; i < n; ++i)
    {
        const float* s = rec + kf * size_t(i);
        float*       d = h.data() + 16 * size_t(i);
        d[0] = s[0], d[1] = s[1], d[2] = s[2];
        d[4] = s[3], d[5] = s[4], d[6] = s[5];
        d[8] = s[6], d[9] = s[7], d[10] = s[8];
        d[12] = s[9], d[13] = s[10], d[14] = s[11];
        d[3]  = kf == 14 ? s[12] : 1.0f;
        d[15] = kf == 14 ? s[13] : 0.0f;
    }
    CL_TRY(rec_.alloc(h.size() * 4, err));
    CL_CUDA(cudaMemcpyAsync(rec_.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st_), err);
    CL_CUDA(cudaMemcpyAsync(scal_.as<unsigned char>() + 16, &n, 4, cudaMemcpyHostToDevice, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::computeGradient(const float4* rec, const uint32_t* count, std::string* err)
{
    CL_CUDA(cudaMemsetAsync(scal_.p, 0, 16, st_), err);
    CL_CUDA(cudaMemsetAsync(scal_.as<double>() + 3, 0, 8, st_), err);
    CL_CUDA(cudaMemsetAsync(trainErr(), 0, 4, st_), err);
    TrainArgs a;
    a.rec       = rec;
    a.count     = count;
    a.batch     = cfg_.batch;
    a.g         = grid();
    a.wt        = wt_.as<const uint4>();
    a.gradTable = reinterpret_cast<float2*>(grad_.f());
    a.gradMlp   = grad_.f() + hashParams_;
    a.err       = trainErr();
    a.enc       = enc_.as<uint4>();
    a.aux       = aux_.as<float4>();
    a.scal      = scal_.as<double>();
    a.learnSel  = cfg_.learn_selection ? 1 : 0;
    a.clamp     = cfg_.weight_clamp;
    kTrainPrep<<<numSMs_ * 2, 256, 0, st_>>>(a, 0);
    CL_CUDA(cudaGetLastError(), err);
    if (a.clamp > 0.0f)
    {
        kTrainPrep<<<numSMs_ * 2, 256, 0, st_>>>(a, 3);
        CL_CUDA(cudaGetLastError(), err);
    }
    const uint32_t tiles = (cfg_.batch + kTcRows - 1) / kTcRows;
    kTrainEncode<<<gridFor(size_t(tiles) * kTcRows, 256, numSMs_ * 8), 256, 0, st_>>>(a);
    CL_CUDA(cudaGetLastError(), err);
    kTrainTc<S, L><<<std::min<uint32_t>(tiles, uint32_t(numSMs_)), kTrainThreads, TrainTc<S>::kSmem, st_>>>(a);
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::trainDevice(const float4* rec, const uint32_t* count, std::string* err)
{
    CL_TRY(computeGradient(rec, count, err));
    ++step_;
    const float    c1 = float(1.0 - std::pow(double(cfg_.beta1), double(step_)));
    const float    c2 = float(1.0 - std::pow(double(cfg_.beta2), double(step_)));
    const uint64_t n4 = paramCount() / 4;
    AdamK          k{cfg_.beta1, cfg_.beta2, cfg_.epsilon, cfg_.learning_rate / c1, 1.0f / c2};
    kAdam<<<gridFor(n4 / 2, 256, numSMs_ * 8), 256, 0, st_>>>(params_.as<float4>(), grad_.as<float4>(),
                                                              m_.as<float4>(), v_.as<float4>(), n4, hashParams_ / 4, k,
                                                              table_.as<uint2>());
    CL_CUDA(cudaGetLastError(), err);
    kFrags<S><<<(fragThreads<S>() + 255) / 256, 256, 0, st_>>>(params_.f() + hashParams_, wt_.as<uint4>());
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

template <class S, class L>
cl_status HashNet<S, L>::gradient(const float* rec, uint32_t n, double* loss, float* grad, std::string* err)
{
    if (!grad || !loss)
    {
        *err = "network: null output";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(upload(rec, n, err));
    const uint32_t* cnt = reinterpret_cast<const uint32_t*>(scal_.as<unsigned char>() + 16);
    CL_TRY(computeGradient(rec_.as<const float4>(), cnt, err));
    CL_CUDA(cudaMemcpyAsync(grad, grad_.p, paramCount() * 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaMemcpyAsync(loss, scal_.as<double>() + 1, 8, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaMemsetAsync(grad_.p, 0, paramCount() * 4, st_), err);
    return checkTrainErr(err);
}

template <class S, class L>
cl_status HashNet<S, L>::trainStepHost(const float* rec, uint32_t n, double* loss, std::string* err)
{
    CL_TRY(upload(rec, n, err));
    const uint32_t* cnt = reinterpret_cast<const uint32_t*>(scal_.as<unsigned char>() + 16);
    CL_TRY(trainDevice(rec_.as<const float4>(), cnt, err));
    if (loss) CL_CUDA(cudaMemcpyAsync(loss, scal_.as<double>() + 1, 8, cudaMemcpyDeviceToHost, st_), err);
    return checkTrainErr(err);
}

// Synchronises the stream and reports a training kernel's timeout.
template <class S, class L> cl_status HashNet<S, L>::checkTrainErr(std::string* err)
{
    uint32_t hf = 0u;
    CL_CUDA(cudaMemcpyAsync(&hf, trainErr(), 4, cudaMemcpyDeviceToHost, st_), err);
    CL_CUDA(cudaStreamSynchronize(st_), err);
    if (hf & kTcTimeout)
    {
        markTcSuspect();
        *err = "network training: a tensor-core wait ran out";
        return CL_ERR_TIMEOUT;
    }
    return CL_OK;
}

template class HashNet<GuideShape, GuideLoss>;
template class HashNet<CacheShape, CacheLoss>;

} // namespace clb
