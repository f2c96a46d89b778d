// Neural path guiding network, device side (no counterpart in the reference
// renderer): multiresolution hash grid + one-blob encoding, a 96-64-64-64-64-48
// ReLU MLP with BF16 operands and FP32 accumulation on the tensor cores, and a
// head of 8 von Mises-Fisher lobes.  The radiance cache uses the same encoding
// and a 96-64-64-16 MLP.  The tensor-core passes (tcgen05, inference and
// training) are in cl_mlp_tc.cuh and cl_guide.cu.
#pragma once

#include "cl_device.cuh"

#include <cuda_bf16.h>

namespace clb
{
namespace guide
{
constexpr int kLevels = 16, kFeat = 2, kHashF = 32, kBlob = 16, kIn = 96, kWidth = 64, kLobes = 8;
constexpr float kKappaMin = -5.0f, kKappaMax = 7.0f;
constexpr float kSelMin = 0.05f, kSelMax = 0.95f; // learned guide-selection probability range
constexpr int   kSelOut = 5 * kLobes;           // head output of its logit

// Network shape: 96 encoded inputs -> 64 (layer 0) -> NH hidden layers of
// 64 -> NO outputs (a multiple of 16), ReLU between layers, no biases.  W_l
// is [out][in] row-major in the flat parameter block.
template <int NH, int NO> struct MlpShape
{
    static_assert(NO % 16 == 0 && NH >= 1, "outputs: a multiple of 16; at least one hidden layer");
    static constexpr int kHidden = NH, kLayers = NH + 2, kOut = NO;
    __host__ __device__ static constexpr int in(int l) { return l == 0 ? kIn : kWidth; }
    __host__ __device__ static constexpr int out(int l) { return l == NH + 1 ? NO : kWidth; }
    __host__ __device__ static constexpr int woff(int l) { return l == 0 ? 0 : kIn * kWidth + (l - 1) * kWidth * kWidth; }
    static constexpr int kParams = kIn * kWidth + NH * kWidth * kWidth + kWidth * NO;
};
// The guiding network (4 hidden layers, 48 outputs: 8 vMF lobes + selection)
// and the radiance cache (2 hidden layers, RGB in the first 3 of 16 outputs).
using GuideShape = MlpShape<3, 48>;
using CacheShape = MlpShape<1, 16>;
constexpr int kOut       = GuideShape::kOut;
constexpr int kMlpParams = GuideShape::kParams; // 21504

// Hash grid: table[l * T + index] holds the 2 features of an entry.
struct GridView
{
    const __nv_bfloat162* __restrict__ table;
    uint32_t mask;      // T - 1
    uint32_t log2T;
    uint32_t denseMask; // bit l: level l is indexed densely ((res+1)^3 <= T)
    uint32_t res[kLevels];
};

// Cell and interpolation weights of level l for p in [0,1]^3 (clamped): the
// cell index is clamped to res-1 so that p = 1 interpolates with weight 1.
struct Cell
{
    uint32_t x, y, z;
    float    wx, wy, wz;
};
__device__ __forceinline__ Cell gridCell(uint32_t res, f3 p)
{
    const float fr = float(res), top = float(res - 1u);
    float       x = p.x * fr, y = p.y * fr, z = p.z * fr;
    float       ix = fminf(floorf(x), top), iy = fminf(floorf(y), top), iz = fminf(floorf(z), top);
    return {uint32_t(ix), uint32_t(iy), uint32_t(iz), x - ix, y - iy, z - iz};
}
// The 8 corner weights, corner k's the product (a b) d of a = wx or 1 - wx,
// b = wy or 1 - wy, d = wz or 1 - wz by bits 0, 1, 2 of k; the 4 products
// a b are shared by the two z layers.
__device__ __forceinline__ void cornerWeights(const Cell& c, float (&w)[8])
{
    const float ax[2] = {1.0f - c.wx, c.wx}, by[2] = {1.0f - c.wy, c.wy}, dz[2] = {1.0f - c.wz, c.wz};
    float       ab[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) ab[k] = ax[k & 1] * by[k >> 1];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = ab[k & 3] * dz[k >> 2];
}
// The 8 corner indices of level l (corner k: +1 along x, y, z for bits 0, 1,
// 2 of k).  A dense level indexes x + r1 (y + r1 z) (r1 = res + 1), so the
// corners add 1, r1 and r1^2 to the cell's index; a hashed level indexes
// (x ^ y P1 ^ z P2) & (T - 1) with P1 = 2654435761, P2 = 805459861 (Mueller
// et al. 2022), built from the per-axis terms, (y + 1) P1 = y P1 + P1 (mod
// 2^32).  The dense/hashed choice depends on the level only, so it is uniform
// across a warp.
__device__ __forceinline__ void cornerIndices(const GridView& g, int l, const Cell& c, uint32_t (&idx)[8])
{
    if ((g.denseMask >> l) & 1u)
    {
        const uint32_t r1 = g.res[l] + 1u, b = c.x + r1 * (c.y + r1 * c.z), b4 = b + r1 * r1;
        idx[0] = b;
        idx[1] = b + 1u;
        idx[2] = b + r1;
        idx[3] = b + r1 + 1u;
        idx[4] = b4;
        idx[5] = b4 + 1u;
        idx[6] = b4 + r1;
        idx[7] = b4 + r1 + 1u;
    }
    else
    {
        const uint32_t y[2] = {c.y * 2654435761u, c.y * 2654435761u + 2654435761u};
        const uint32_t z[2] = {c.z * 805459861u, c.z * 805459861u + 805459861u};
#pragma unroll
        for (int k = 0; k < 8; ++k) idx[k] = ((c.x + uint32_t(k & 1)) ^ y[(k >> 1) & 1] ^ z[k >> 2]) & g.mask;
    }
}
__device__ __forceinline__ f3 clampUnit(f3 p)
{
    return {fminf(fmaxf(p.x, 0.0f), 1.0f), fminf(fmaxf(p.y, 0.0f), 1.0f), fminf(fmaxf(p.z, 0.0f), 1.0f)};
}
// Trilinear features of level l (8 independent 4-byte gathers).
__device__ __forceinline__ float2 encodeLevel(const GridView& g, int l, f3 p)
{
    const Cell                          c  = gridCell(g.res[l], p);
    const __nv_bfloat162* __restrict__ tl = g.table + (size_t(l) << g.log2T);
    uint32_t                            idx[8];
    cornerIndices(g, l, c, idx);
    __nv_bfloat162 t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = __ldg(tl + idx[k]);
    float w[8];
    cornerWeights(c, w);
    float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        float2 v = __bfloat1622float2(t[k]);
        f0       = fmaf(w[k], v.x, f0);
        f1       = fmaf(w[k], v.y, f1);
    }
    return {f0, f1};
}

// One-blob encoding of a direction: theta/pi and phi/(2 pi) + 1/2, 16
// Gaussian bins each (sigma 1/16) - the 32 bf16 values go to dst[0..31].
// The bins use the fast hardware exponential (__expf): its error is far
// below the BF16 rounding that follows, and the IEEE expf cost 5% of the
// guide's fused inference.
__device__ __forceinline__ void oneBlob(f3 d, __nv_bfloat16* dst)
{
    float th = acosf(fminf(fmaxf(d.z, -1.0f), 1.0f)) * kInvPi;
    float ph = atan2f(d.y, d.x) * (0.5f * kInvPi) + 0.5f;
#pragma unroll
    for (int i = 0; i < kBlob; ++i)
    {
        float c  = (float(i) + 0.5f) * (1.0f / kBlob);
        float a  = th - c, b = ph - c;
        dst[i]         = __float2bfloat16_rn(__expf(-a * a * 128.0f));
        dst[kBlob + i] = __float2bfloat16_rn(__expf(-b * b * 128.0f));
    }
}

// The same encoding as 16 packed bf16 pairs (register-resident rows).
__device__ __forceinline__ void oneBlobPacked(f3 d, uint32_t* dst)
{
    float th = acosf(fminf(fmaxf(d.z, -1.0f), 1.0f)) * kInvPi;
    float ph = atan2f(d.y, d.x) * (0.5f * kInvPi) + 0.5f;
#pragma unroll
    for (int i = 0; i < kBlob; i += 2)
    {
        float c0 = (float(i) + 0.5f) * (1.0f / kBlob), c1 = (float(i) + 1.5f) * (1.0f / kBlob);
        float a0 = th - c0, a1 = th - c1, b0 = ph - c0, b1 = ph - c1;
        __nv_bfloat162 t = __floats2bfloat162_rn(__expf(-a0 * a0 * 128.0f), __expf(-a1 * a1 * 128.0f));
        __nv_bfloat162 u = __floats2bfloat162_rn(__expf(-b0 * b0 * 128.0f), __expf(-b1 * b1 * 128.0f));
        dst[i / 2]             = *reinterpret_cast<uint32_t*>(&t);
        dst[(kBlob + i) / 2]   = *reinterpret_cast<uint32_t*>(&u);
    }
}

// Encoded input row of one sample: 32 hash features, one-blob of n and wo.
__device__ __forceinline__ void encodeRow(const GridView& g, f3 p, f3 n, f3 wo, __nv_bfloat16* row)
{
    p = clampUnit(p);
#pragma unroll 4
    for (int l = 0; l < kLevels; ++l)
    {
        float2 f = encodeLevel(g, l, p);
        *reinterpret_cast<__nv_bfloat162*>(row + 2 * l) = __floats2bfloat162_rn(f.x, f.y);
    }
    oneBlob(n, row + kHashF);
    oneBlob(wo, row + kHashF + 2 * kBlob);
}
__device__ __forceinline__ void zeroRow(__nv_bfloat16* row)
{
    uint32_t* r = reinterpret_cast<uint32_t*>(row);
#pragma unroll
    for (int i = 0; i < kIn / 2; ++i) r[i] = 0u;
}

// ---------------------------------------------------------------------------
// BF16 packing
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float reluF(float x) { return x > 0.0f ? x : 0.0f; }

// ---------------------------------------------------------------------------
// vMF mixture head
// ---------------------------------------------------------------------------
struct Lobes
{
    float4 l[kLobes]; // {mu.xyz, kappa}
    float  w[kLobes]; // weights; they sum to the probability of sampling the guide
};

__device__ __forceinline__ float selectionProb(float logit)
{
    return kSelMin + (kSelMax - kSelMin) / (1.0f + expf(-logit));
}

// Lobe parameters from the head outputs o[5k..5k+4] = (mu_xyz, log kappa,
// weight logit); the weights are normalised to `alpha`, the probability of
// sampling the guide (alpha < 0: learned, from output 40).
__device__ __forceinline__ void headLobes(const float* o, Lobes* L, float alpha = 1.0f)
{
    if (alpha < 0.0f) alpha = selectionProb(o[kSelOut]);
    float mx = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        float e = expf(o[5 * k + 4] - mx);
        L->w[k] = e;
        s += e;
    }
    const float inv = alpha / s;
#pragma unroll
    for (int k = 0; k < kLobes; ++k)
    {
        float x = o[5 * k], y = o[5 * k + 1], z = o[5 * k + 2];
        float rn  = 1.0f / fmaxf(sqrtf(x * x + y * y + z * z), 1e-6f);
        float kap = expf(fminf(fmaxf(o[5 * k + 3], kKappaMin), kKappaMax));
        L->l[k]   = make_float4(x * rn, y * rn, z * rn, kap);
        L->w[k] *= inv;
    }
}

// vMF density kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (mu.d - 1)}.
__device__ __forceinline__ float vmfPdf(float4 l, f3 d)
{
    float c = l.x * d.x + l.y * d.y + l.z * d.z;
    return l.w / (2.0f * kPiF * -expm1f(-2.0f * l.w)) * expf(l.w * (c - 1.0f));
}

__device__ __forceinline__ float mixturePdf(const Lobes& L, f3 d)
{
    float p = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) p = fmaf(L.w[k], vmfPdf(L.l[k], d), p);
    return p;
}

// Orthonormal basis around n (Duff et al. 2017).
__device__ __forceinline__ void onb(f3 n, f3* t, f3* b)
{
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a    = -1.0f / (sign + n.z);
    float bb   = n.x * n.y * a;
    *t         = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
    *b         = {bb, sign + n.y * n.y * a, -n.y};
}

// Lobe by u0 in [0, sum of weights) over the weights' CDF; direction by
// Jakob's inversion (2012):
// w = 1 + log(u1 + (1 - u1) e^{-2 kappa}) / kappa, phi = 2 pi u2.
__device__ __forceinline__ f3 mixtureSample(const Lobes& L, float u0, float u1, float u2)
{
    int   k   = kLobes - 1;
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j)
    {
        acc += L.w[j];
        if (u0 < acc && k == kLobes - 1 && j < kLobes - 1) k = j;
    }
    // First lobe whose running sum exceeds u0 (kept branch-free above).
    float4 l   = L.l[0];
#pragma unroll
    for (int j = 1; j < kLobes; ++j)
        if (j == k) l = L.l[j];
    float kap = l.w;
    float w   = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kap)) / kap;
    w         = fminf(fmaxf(w, -1.0f), 1.0f);
    float s   = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float sp, cp;
    sincosf(2.0f * kPiF * u2, &sp, &cp);
    f3 t, b, mu{l.x, l.y, l.z};
    onb(mu, &t, &b);
    f3 d = w * mu + (s * cp) * t;
    d    = d + (s * sp) * b;
    return d;
}

} // namespace guide
} // namespace clb
