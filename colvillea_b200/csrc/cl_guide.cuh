// Neural path guiding network, device side (no counterpart in the reference
// renderer): multiresolution hash grid + one-blob encoding, a 96-64-64-64-64-48
// ReLU MLP with BF16 operands and FP32 accumulation on the tensor cores, and a
// head of 8 von Mises-Fisher lobes.
//
// Tensor-core mapping (mma.sync m16n8k16, BF16 in, FP32 accumulate): a warp
// owns 16-row tiles of samples.  The accumulator fragment of two adjacent
// 8-column tiles is exactly the A fragment of one 16-column k-tile of the next
// layer, so activations stay in registers from layer to layer; only the input
// encoding (one shared-memory tile per warp) and the weights (fragment-ordered
// in shared memory, one 8-byte load per lane per fragment) are read from
// shared memory.
#pragma once

#include "cl_device.cuh"

#include <cuda_bf16.h>

namespace clb
{
namespace guide
{
constexpr int kLevels = 16, kFeat = 2, kHashF = 32, kBlob = 16, kIn = 96, kWidth = 64, kLobes = 8;
constexpr int kXS = 104; // encoded-input tile row stride (bf16): 208 B, conflict-free ldmatrix rows
constexpr float kKappaMin = -5.0f, kKappaMax = 7.0f;
constexpr float kSelMin = 0.05f, kSelMax = 0.95f; // learned guide-selection probability range
constexpr int   kSelOut = 5 * kLobes;           // head output of its logit

// Network shape: 96 encoded inputs -> 64 (layer 0) -> NH hidden layers of
// 64 -> NO outputs (a multiple of 16), ReLU between layers, no biases.  W_l
// is [out][in] row-major in the flat parameter block.
//   forward fragments of layer l: (in/16) k-tiles x (out/8) n-tiles;
//   backward fragments: (out/16) k-tiles x (in/8) n-tiles, only the 32
//   hash-grid columns at layer 0 (the one-blob inputs get no gradient).
// Training staging rows: the input of every layer [96 | 64 ...] and the
// output gradient of every layer [64 ... | NO], bf16.
template <int NH, int NO> struct MlpShape
{
    static_assert(NO % 16 == 0 && NH >= 1, "outputs: a multiple of 16; at least one hidden layer");
    static constexpr int kHidden = NH, kLayers = NH + 2, kOut = NO;
    __host__ __device__ static constexpr int in(int l) { return l == 0 ? kIn : kWidth; }
    __host__ __device__ static constexpr int out(int l) { return l == NH + 1 ? NO : kWidth; }
    __host__ __device__ static constexpr int woff(int l) { return l == 0 ? 0 : kIn * kWidth + (l - 1) * kWidth * kWidth; }
    static constexpr int kParams = kIn * kWidth + NH * kWidth * kWidth + kWidth * NO;
    __host__ __device__ static constexpr int fwdNT(int l) { return out(l) / 8; }
    __host__ __device__ static constexpr int bwdNT(int l) { return l == 0 ? kHashF / 8 : in(l) / 8; }
    __host__ __device__ static constexpr int fwdOff(int l) { return l == 0 ? 0 : 48 + (l - 1) * 32; }
    __host__ __device__ static constexpr int bwdOff(int l) { return l == 0 ? 0 : 16 + (l - 1) * 32; }
    static constexpr int kFwdFrags = 48 + NH * 32 + 4 * (NO / 8);
    static constexpr int kBwdFrags = 16 + NH * 32 + (NO / 16) * 8;
    static constexpr int kFwdBytes = kFwdFrags * 32 * 8;
    static constexpr int kBwdBytes = kBwdFrags * 32 * 8;
    static constexpr int kActRow   = kIn + (NH + 1) * kWidth;
    static constexpr int kDeltaRow = (NH + 1) * kWidth + NO;
    __host__ __device__ static constexpr int actOff(int l) { return l == 0 ? 0 : kIn + (l - 1) * kWidth; }
    __host__ __device__ static constexpr int deltaOff(int l) { return l * kWidth; }
    static constexpr int kOS = NO + 1; // output tile row stride (f32)
    static constexpr int kDS = NO + 8; // output-gradient tile row stride (bf16), conflict-free ldmatrix rows
};
// The guiding network (4 hidden layers, 48 outputs: 8 vMF lobes + selection)
// and the radiance cache (2 hidden layers, RGB in the first 3 of 16 outputs).
using GuideShape = MlpShape<3, 48>;
using CacheShape = MlpShape<1, 16>;
constexpr int kOut          = GuideShape::kOut;
constexpr int kOS           = GuideShape::kOS;
constexpr int kMlpParams    = GuideShape::kParams;   // 21504
constexpr int kFwdFragBytes = GuideShape::kFwdBytes;

// Hash grid: table[l * T + index] holds the 2 features of an entry.
struct GridView
{
    const __nv_bfloat162* __restrict__ table;
    uint32_t mask;      // T - 1
    uint32_t log2T;
    uint32_t denseMask; // bit l: level l is indexed densely ((res+1)^3 <= T)
    uint32_t res[kLevels];
};

__device__ __forceinline__ uint32_t gridIndex(uint32_t x, uint32_t y, uint32_t z, uint32_t r1, bool dense,
                                              uint32_t mask)
{
    if (dense) return x + r1 * (y + r1 * z);
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & mask;
}

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
__device__ __forceinline__ float cornerWeight(const Cell& c, int k)
{
    float a = (k & 1) ? c.wx : 1.0f - c.wx;
    float b = (k & 2) ? c.wy : 1.0f - c.wy;
    float d = (k & 4) ? c.wz : 1.0f - c.wz;
    return a * b * d;
}
__device__ __forceinline__ uint32_t cornerIndex(const GridView& g, int l, const Cell& c, int k)
{
    const uint32_t r1 = g.res[l] + 1u;
    return gridIndex(c.x + (k & 1), c.y + ((k >> 1) & 1), c.z + ((k >> 2) & 1), r1, (g.denseMask >> l) & 1u, g.mask);
}
__device__ __forceinline__ f3 clampUnit(f3 p)
{
    return {fminf(fmaxf(p.x, 0.0f), 1.0f), fminf(fmaxf(p.y, 0.0f), 1.0f), fminf(fmaxf(p.z, 0.0f), 1.0f)};
}
// Trilinear features of level l (8 independent 4-byte gathers).
__device__ __forceinline__ float2 encodeLevel(const GridView& g, int l, f3 p)
{
    Cell           c    = gridCell(g.res[l], p);
    const size_t   base = size_t(l) << g.log2T;
    uint32_t       idx[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) idx[k] = cornerIndex(g, l, c, k);
    __nv_bfloat162 t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = __ldg(g.table + base + idx[k]);
    float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        float  w = cornerWeight(c, k);
        float2 v = __bfloat1622float2(t[k]);
        f0       = fmaf(w, v.x, f0);
        f1       = fmaf(w, v.y, f1);
    }
    return {f0, f1};
}

// One-blob encoding of a direction: theta/pi and phi/(2 pi) + 1/2, 16
// Gaussian bins each (sigma 1/16) - the 32 bf16 values go to dst[0..31].
__device__ __forceinline__ void oneBlob(f3 d, __nv_bfloat16* dst)
{
    float th = acosf(fminf(fmaxf(d.z, -1.0f), 1.0f)) * kInvPi;
    float ph = atan2f(d.y, d.x) * (0.5f * kInvPi) + 0.5f;
#pragma unroll
    for (int i = 0; i < kBlob; ++i)
    {
        float c  = (float(i) + 0.5f) * (1.0f / kBlob);
        float a  = th - c, b = ph - c;
        dst[i]         = __float2bfloat16_rn(expf(-a * a * 128.0f));
        dst[kBlob + i] = __float2bfloat16_rn(expf(-b * b * 128.0f));
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
        __nv_bfloat162 t = __floats2bfloat162_rn(expf(-a0 * a0 * 128.0f), expf(-a1 * a1 * 128.0f));
        __nv_bfloat162 u = __floats2bfloat162_rn(expf(-b0 * b0 * 128.0f), expf(-b1 * b1 * 128.0f));
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
// Tensor-core primitives
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float reluF(float x) { return x > 0.0f ? x : 0.0f; }

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const void* p)
{
    uint32_t a = uint32_t(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], const void* p)
{
    uint32_t a = uint32_t(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// A fragments of one 16-row tile whose rows start at `tile` (stride `ld`
// bf16), k-tile kt: lane l addresses row l & 15, column 16 kt + 8 (l >> 4).
__device__ __forceinline__ void loadA(uint32_t (&a)[4], const __nv_bfloat16* tile, int ld, int kt, uint32_t lane)
{
    ldsm4(a, tile + (lane & 15u) * ld + kt * 16 + (lane >> 4) * 8);
}

// Accumulators of n-tiles 2j, 2j+1 -> A fragment of k-tile j (after ReLU).
__device__ __forceinline__ void accToA(const float (&c0)[4], const float (&c1)[4], uint32_t (&a)[4])
{
    a[0] = packBf16(reluF(c0[0]), reluF(c0[1]));
    a[1] = packBf16(reluF(c0[2]), reluF(c0[3]));
    a[2] = packBf16(reluF(c1[0]), reluF(c1[1]));
    a[3] = packBf16(reluF(c1[2]), reluF(c1[3]));
}

// Hidden layer from registers: in (4 k-tiles) -> out (8 n-tiles) -> ReLU.
template <int MT>
__device__ __forceinline__ void hiddenLayer(const uint2* __restrict__ wf, const uint32_t (&in)[MT][4][4],
                                            uint32_t (&out)[MT][4][4], uint32_t lane)
{
    float acc[MT][8][4];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int n = 0; n < 8; ++n) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
        {
            uint2 b = wf[(kt * 8 + nt) * 32 + lane];
#pragma unroll
            for (int m = 0; m < MT; ++m) mma16816(acc[m][nt], in[m][kt], b.x, b.y);
        }
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int j = 0; j < 4; ++j) accToA(acc[m][2 * j], acc[m][2 * j + 1], out[m][j]);
}

// Layer 0: the encoded-input tile (MT*16 rows, stride kXS, shared memory)
// -> ReLU activations as A fragments.
template <int MT>
__device__ __forceinline__ void inputLayer(const uint2* __restrict__ wf, const __nv_bfloat16* x, uint32_t lane,
                                           uint32_t (&h)[MT][4][4])
{
    float acc[MT][8][4];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int n = 0; n < 8; ++n) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 6; ++kt)
    {
        uint32_t a[MT][4];
#pragma unroll
        for (int m = 0; m < MT; ++m) loadA(a[m], x + m * 16 * kXS, kXS, kt, lane);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
        {
            uint2 b = wf[(kt * 8 + nt) * 32 + lane];
#pragma unroll
            for (int m = 0; m < MT; ++m) mma16816(acc[m][nt], a[m], b.x, b.y);
        }
    }
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int j = 0; j < 4; ++j) accToA(acc[m][2 * j], acc[m][2 * j + 1], h[m][j]);
}

// Last layer: 64 inputs (A fragments) -> NO/8 n-tiles of FP32 outputs.
template <class S, int MT>
__device__ __forceinline__ void outputLayer(const uint2* __restrict__ wl, const uint32_t (&in)[MT][4][4],
                                            float (&out)[MT][S::kOut / 8][4], uint32_t lane)
{
    constexpr int NT = S::kOut / 8;
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int n = 0; n < NT; ++n) out[m][n][0] = out[m][n][1] = out[m][n][2] = out[m][n][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
        {
            uint2 b = wl[(kt * NT + nt) * 32 + lane];
#pragma unroll
            for (int m = 0; m < MT; ++m) mma16816(out[m][nt], in[m][kt], b.x, b.y);
        }
}

// Forward pass of MT 16-row tiles.  `x`: the warp's encoded-input tile;
// `wf`: forward fragments (shared memory).  h[l]: A fragments of the input
// of layer l+1, kept for the backward pass; out: the outputs' accumulators.
template <class S, int MT>
__device__ __forceinline__ void mlpForward(const uint2* __restrict__ wf, const __nv_bfloat16* x, uint32_t lane,
                                           uint32_t (&h)[S::kHidden + 1][MT][4][4], float (&out)[MT][S::kOut / 8][4])
{
    inputLayer<MT>(wf, x, lane, h[0]);
#pragma unroll
    for (int l = 1; l <= S::kHidden; ++l) hiddenLayer<MT>(wf + S::fwdOff(l) * 32, h[l - 1], h[l], lane);
    outputLayer<S, MT>(wf + S::fwdOff(S::kHidden + 1) * 32, h[S::kHidden], out, lane);
}

// Inference-only forward (activations ping-pong between two register sets).
template <class S, int MT>
__device__ __forceinline__ void mlpInfer(const uint2* __restrict__ wf, const __nv_bfloat16* x, uint32_t lane,
                                         float (&out)[MT][S::kOut / 8][4])
{
    uint32_t ha[MT][4][4], hb[MT][4][4];
    inputLayer<MT>(wf, x, lane, ha);
#pragma unroll
    for (int l = 1; l <= S::kHidden; ++l)
    {
        if (l & 1)
            hiddenLayer<MT>(wf + S::fwdOff(l) * 32, ha, hb, lane);
        else
            hiddenLayer<MT>(wf + S::fwdOff(l) * 32, hb, ha, lane);
    }
    if (S::kHidden & 1)
        outputLayer<S, MT>(wf + S::fwdOff(S::kHidden + 1) * 32, hb, out, lane);
    else
        outputLayer<S, MT>(wf + S::fwdOff(S::kHidden + 1) * 32, ha, out, lane);
}

// Output accumulators -> rows of a float tile (stride S::kOS).
template <class S, int MT>
__device__ __forceinline__ void storeOut(const float (&out)[MT][S::kOut / 8][4], float* tile, uint32_t lane)
{
    const uint32_t g = lane >> 2, t = lane & 3u;
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int n = 0; n < S::kOut / 8; ++n)
        {
            float* r0 = tile + (m * 16 + g) * S::kOS + n * 8 + 2 * t;
            float* r1 = r0 + 8 * S::kOS;
            r0[0]     = out[m][n][0];
            r0[1]     = out[m][n][1];
            r1[0]     = out[m][n][2];
            r1[1]     = out[m][n][3];
        }
}

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
        float n = fmaxf(sqrtf(x * x + y * y + z * z), 1e-6f);
        float kap = expf(fminf(fmaxf(o[5 * k + 3], kKappaMin), kKappaMax));
        L->l[k]   = make_float4(x / n, y / n, z / n, kap);
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
