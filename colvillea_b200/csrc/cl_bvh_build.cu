// Device build of the 8-wide compressed BVH (layout in cl_bvh.cuh).
//
// Replaces OptiX's BLAS/TLAS builds (owlGroupBuildAccel,
// src/core/devices/optixdevice.cpp:136-233) with a hand-written builder:
//   1. per-triangle boxes and centroid bounds;
//   2. 63-bit Morton codes of the centroids, sorted (CUB radix sort);
//   3. binary tree by PLOC clustering over the Morton order (Meister and
//      Bittner 2018), SAH-quality at LBVH speed; the binary radix tree of
//      Karras (HPG 2012) with bottom-up boxes is kept as a fallback;
//   4. surface-area-optimal collapse to 8-wide nodes (Ylitie, Karras and
//      Laine, HPG 2017): slot costs bottom up over the binary tree, then one
//      level of wide nodes per launch, each taking the children that the
//      costs' minima give it; subtrees of at most 3 triangles become leaf
//      slots; slots are assigned by octant; child boxes are quantised to
//      8 bits per plane, rounded outwards around a widened parent box.
#include "cl_bvh.cuh"
#include "cl_internal.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <vector>

namespace clb
{
namespace
{
constexpr uint32_t kLeafFlag = 0x80000000u;

__device__ __forceinline__ uint32_t fordered(float f)
{
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float funordered(uint32_t b)
{
    return __uint_as_float((b & 0x80000000u) ? (b & 0x7fffffffu) : ~b);
}

// Widening of every child box before quantisation: 2^-20 of the scene
// scale (the product is exact, so host and device agree bit for bit).
__host__ __device__ inline float sceneMargin(const float lo[3], const float hi[3])
{
    float scale = 0.0f;
    for (int a = 0; a < 3; ++a)
    {
        scale = fmaxf(scale, fmaxf(fabsf(lo[a]), fabsf(hi[a])));
        scale = fmaxf(scale, hi[a] - lo[a]);
    }
    return scale * 9.5367431640625e-07f + 1e-30f;
}

struct Bounds
{
    uint32_t clo[3], chi[3]; // centroid bounds (ordered ints)
    uint32_t slo[3], shi[3]; // scene bounds
};

__global__ void kTriBounds(const float* __restrict__ tri9, uint32_t n, float* __restrict__ lo, float* __restrict__ hi,
                           Bounds* b)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float    c[3], l[3], h[3];
    bool     valid = i < n;
    if (valid)
    {
        const float* t = tri9 + 9 * size_t(i);
        for (int a = 0; a < 3; ++a)
        {
            l[a] = fminf(fminf(t[a], t[3 + a]), t[6 + a]);
            h[a] = fmaxf(fmaxf(t[a], t[3 + a]), t[6 + a]);
            c[a] = 0.5f * l[a] + 0.5f * h[a];
            lo[3 * size_t(i) + a] = l[a];
            hi[3 * size_t(i) + a] = h[a];
        }
    }
    for (int a = 0; a < 3; ++a)
    {
        uint32_t cl = valid ? fordered(c[a]) : 0xffffffffu, ch = valid ? fordered(c[a]) : 0u;
        uint32_t sl = valid ? fordered(l[a]) : 0xffffffffu, sh = valid ? fordered(h[a]) : 0u;
        for (int o = 16; o > 0; o >>= 1)
        {
            cl = min(cl, __shfl_xor_sync(0xffffffffu, cl, o));
            ch = max(ch, __shfl_xor_sync(0xffffffffu, ch, o));
            sl = min(sl, __shfl_xor_sync(0xffffffffu, sl, o));
            sh = max(sh, __shfl_xor_sync(0xffffffffu, sh, o));
        }
        if ((threadIdx.x & 31) == 0)
        {
            atomicMin(&b->clo[a], cl);
            atomicMax(&b->chi[a], ch);
            atomicMin(&b->slo[a], sl);
            atomicMax(&b->shi[a], sh);
        }
    }
}

__device__ __forceinline__ uint64_t expand21(uint32_t v)
{
    uint64_t x = v & 0x1fffffu;
    x          = (x | x << 32) & 0x1f00000000ffffull;
    x          = (x | x << 16) & 0x1f0000ff0000ffull;
    x          = (x | x << 8) & 0x100f00f00f00f00full;
    x          = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x          = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void kMorton(const float* __restrict__ lo, const float* __restrict__ hi, uint32_t n, const Bounds* b,
                        uint64_t* __restrict__ keys, uint32_t* __restrict__ ids)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
    for (int a = 0; a < 3; ++a)
    {
        float cmin = funordered(b->clo[a]), cmax = funordered(b->chi[a]);
        float c    = 0.5f * lo[3 * size_t(i) + a] + 0.5f * hi[3 * size_t(i) + a];
        float ext  = cmax - cmin;
        float u    = ext > 0.0f ? (c - cmin) / ext : 0.5f;
        u          = fminf(fmaxf(u, 0.0f), 1.0f);
        q[a]       = min(uint32_t(u * 2097152.0f), 2097151u);
    }
    keys[i] = expand21(q[0]) | (expand21(q[1]) << 1) | (expand21(q[2]) << 2);
    ids[i]  = i;
}

__device__ __forceinline__ int delta(const uint64_t* keys, int n, int i, int j)
{
    if (j < 0 || j > n - 1) return -1;
    uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clzll(a ^ b);
}

__global__ void kRadixTree(const uint64_t* __restrict__ keys, int n, uint32_t* __restrict__ left,
                           uint32_t* __restrict__ right, uint32_t* __restrict__ parent)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d    = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j     = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s     = 0;
    int t     = l;
    do
    {
        t = (t + 1) / 2;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int      g  = i + s * d + min(d, 0);
    uint32_t lc = (min(i, j) == g) ? (uint32_t(g) | kLeafFlag) : uint32_t(g);
    uint32_t rc = (max(i, j) == g + 1) ? (uint32_t(g + 1) | kLeafFlag) : uint32_t(g + 1);
    left[i]     = lc;
    right[i]    = rc;
    parent[(lc & kLeafFlag) ? (n - 1 + (lc & ~kLeafFlag)) : lc] = uint32_t(i);
    parent[(rc & kLeafFlag) ? (n - 1 + (rc & ~kLeafFlag)) : rc] = uint32_t(i);
}

__device__ __forceinline__ void refBox(uint32_t ref, const float* lo, const float* hi, const uint32_t* ids,
                                       const float* nlo, const float* nhi, float* l, float* h)
{
    if (ref & kLeafFlag)
    {
        uint32_t t = ids[ref & ~kLeafFlag];
        for (int a = 0; a < 3; ++a)
        {
            l[a] = lo[3 * size_t(t) + a];
            h[a] = hi[3 * size_t(t) + a];
        }
    }
    else
        for (int a = 0; a < 3; ++a)
        {
            l[a] = __ldcg(nlo + 3 * size_t(ref) + a);
            h[a] = __ldcg(nhi + 3 * size_t(ref) + a);
        }
}

__global__ void kBottomUp(int n, const float* __restrict__ lo, const float* __restrict__ hi, const uint32_t* __restrict__ ids,
                          const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                          const uint32_t* __restrict__ parent, float* nlo, float* nhi, uint32_t* count,
                          uint32_t* arrive)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t node = parent[n - 1 + j];
    while (node != 0xffffffffu)
    {
        __threadfence();
        if (atomicAdd(&arrive[node], 1u) == 0u) return;
        __threadfence();
        float    l0[3], h0[3], l1[3], h1[3];
        uint32_t a = left[node], b = right[node];
        refBox(a, lo, hi, ids, nlo, nhi, l0, h0);
        refBox(b, lo, hi, ids, nlo, nhi, l1, h1);
        for (int k = 0; k < 3; ++k)
        {
            nlo[3 * size_t(node) + k] = fminf(l0[k], l1[k]);
            nhi[3 * size_t(node) + k] = fmaxf(h0[k], h1[k]);
        }
        uint32_t ca = (a & kLeafFlag) ? 1u : __ldcg(count + a);
        uint32_t cb = (b & kLeafFlag) ? 1u : __ldcg(count + b);
        count[node] = ca + cb;
        node        = parent[node];
    }
}

// ---------------------------------------------------------------------------
// PLOC (Meister and Bittner, "Parallel Locally-Ordered Clustering for
// Bounding Volume Hierarchy Construction", IEEE TVCG 2018).  Clusters start as
// the Morton-sorted triangles; each iteration finds every cluster's nearest
// neighbour (smallest merged surface area) within a window of +-kPlocRadius
// positions, merges mutual nearest neighbours into a new inner node and
// compacts the cluster list in order, until one cluster is left.
// ---------------------------------------------------------------------------
constexpr int kPlocRadius = 16;
constexpr int kPlocBlock  = 256;

__device__ __forceinline__ float mergedArea(float4 alo, float4 ahi, float4 blo, float4 bhi)
{
    float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    return dx * dy + dy * dz + dz * dx;
}

__global__ void kPlocInit(uint32_t n, const uint32_t* __restrict__ ids, const float* __restrict__ lo,
                          const float* __restrict__ hi, uint32_t* __restrict__ C, float4* __restrict__ blo,
                          float4* __restrict__ bhi)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t t = ids[i];
    C[i]       = i | kLeafFlag;
    blo[i]     = make_float4(lo[3 * size_t(t)], lo[3 * size_t(t) + 1], lo[3 * size_t(t) + 2], 0.0f);
    bhi[i]     = make_float4(hi[3 * size_t(t)], hi[3 * size_t(t) + 1], hi[3 * size_t(t) + 2], 0.0f);
}

// The cluster count m lives in device memory (mDev), so that iterations run
// without a host round trip; launches are sized for an upper bound of m and
// threads past m return.  With m <= 1 the clustering is done and the
// iteration changes nothing.
__global__ void __launch_bounds__(kPlocBlock) kPlocNearest(const uint32_t* __restrict__ mDev,
                                                           const float4* __restrict__ blo,
                                                           const float4* __restrict__ bhi, uint32_t* __restrict__ nn)
{
    const uint32_t m = *mDev;
    if (m <= 1u) return;
    __shared__ float4 slo[kPlocBlock + 2 * kPlocRadius], shi[kPlocBlock + 2 * kPlocRadius];
    const int b0 = int(blockIdx.x) * kPlocBlock - kPlocRadius;
    for (int k = threadIdx.x; k < kPlocBlock + 2 * kPlocRadius; k += kPlocBlock)
    {
        int g = b0 + k;
        if (g >= 0 && g < int(m))
        {
            slo[k] = blo[g];
            shi[k] = bhi[g];
        }
    }
    __syncthreads();
    int i = int(blockIdx.x) * kPlocBlock + int(threadIdx.x);
    if (i >= int(m)) return;
    int    li = i - b0;
    float4 alo = slo[li], ahi = shi[li];
    float  best  = FLT_MAX;
    int    bestj = i == 0 ? 1 : i - 1;
    int    j0 = max(0, i - kPlocRadius), j1 = min(int(m) - 1, i + kPlocRadius);
    for (int j = j0; j <= j1; ++j)
    {
        if (j == i) continue;
        float c = mergedArea(alo, ahi, slo[j - b0], shi[j - b0]);
        if (c < best)
        {
            best  = c;
            bestj = j;
        }
    }
    nn[i] = uint32_t(bestj);
}

struct PlocTree
{
    uint32_t* left;
    uint32_t* right;
    float*    nlo;
    float*    nhi;
    uint32_t* count;
    uint32_t* nodeCounter;
};

__global__ void kPlocMerge(const uint32_t* __restrict__ mDev, uint32_t mBound, const uint32_t* __restrict__ C,
                           const float4* __restrict__ blo, const float4* __restrict__ bhi,
                           const uint32_t* __restrict__ nn, uint32_t* __restrict__ valid, uint32_t* __restrict__ C2,
                           float4* __restrict__ blo2, float4* __restrict__ bhi2, PlocTree T, uint32_t maxInner)
{
    const uint32_t m = *mDev;
    uint32_t       i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mBound) return;
    if (i >= m || m <= 1u)
    {
        valid[i] = 0u; // outside the live range: the scan over mBound counts nothing here
        return;
    }
    uint32_t j      = nn[i];
    bool     mutual = nn[j] == i;
    if (mutual && j < i)
    {
        valid[i] = 0u; // merged into cluster j
        return;
    }
    valid[i] = 1u;
    if (!mutual)
    {
        C2[i]   = C[i];
        blo2[i] = blo[i];
        bhi2[i] = bhi[i];
        return;
    }
    uint32_t k = atomicAdd(T.nodeCounter, 1u);
    if (k >= maxInner)
    {
        valid[i] = 1u;
        C2[i]    = C[i];
        blo2[i]  = blo[i];
        bhi2[i]  = bhi[i];
        return;
    }
    uint32_t a = C[i], b = C[j];
    float4   lo = make_float4(fminf(blo[i].x, blo[j].x), fminf(blo[i].y, blo[j].y), fminf(blo[i].z, blo[j].z), 0.0f);
    float4   hi = make_float4(fmaxf(bhi[i].x, bhi[j].x), fmaxf(bhi[i].y, bhi[j].y), fmaxf(bhi[i].z, bhi[j].z), 0.0f);
    T.left[k]  = a;
    T.right[k] = b;
    T.nlo[3 * size_t(k)] = lo.x;
    T.nlo[3 * size_t(k) + 1] = lo.y;
    T.nlo[3 * size_t(k) + 2] = lo.z;
    T.nhi[3 * size_t(k)] = hi.x;
    T.nhi[3 * size_t(k) + 1] = hi.y;
    T.nhi[3 * size_t(k) + 2] = hi.z;
    uint32_t ca = (a & kLeafFlag) ? 1u : T.count[a];
    uint32_t cb = (b & kLeafFlag) ? 1u : T.count[b];
    T.count[k]  = ca + cb;
    C2[i]       = k;
    blo2[i]     = lo;
    bhi2[i]     = hi;
}

__global__ void kPlocScatter(const uint32_t* __restrict__ mDev, const uint32_t* __restrict__ valid,
                             const uint32_t* __restrict__ pos, const uint32_t* __restrict__ C2,
                             const float4* __restrict__ blo2, const float4* __restrict__ bhi2,
                             uint32_t* __restrict__ C, float4* __restrict__ blo, float4* __restrict__ bhi)
{
    const uint32_t m = *mDev;
    uint32_t       i = blockIdx.x * blockDim.x + threadIdx.x;
    if (m <= 1u || i >= m || !valid[i]) return;
    uint32_t d = pos[i];
    C[d]       = C2[i];
    blo[d]     = blo2[i];
    bhi[d]     = bhi2[i];
}

// Next iteration's cluster count: the survivors of this one.
__global__ void kPlocCount(const uint32_t* __restrict__ mDev, uint32_t* __restrict__ mNext,
                           const uint32_t* __restrict__ valid, const uint32_t* __restrict__ pos)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t m = *mDev;
    *mNext     = m <= 1u ? m : pos[m - 1] + valid[m - 1];
}

// ---------------------------------------------------------------------------
// Surface-area-optimal collapse (Ylitie, Karras and Laine, "Efficient
// incoherent ray traversal on GPUs through compressed wide BVHs", HPG 2017):
// cost(n, i), i = 1..8, is the smallest surface-area cost of representing the
// binary subtree of n with at most i slots of a wide node.
//   dist(n, j)  = min over k of cost(left, k) + cost(right, j - k)
//   cost(n, 1)  = A(n) c_tri |T(n)|          if |T(n)| <= 3 (a leaf slot)
//               = dist(n, 8) + A(n) c_node   otherwise (a wide node)
//   cost(n, i)  = min(cost(n, i - 1), dist(n, i))
// A triangle costs A(t) c_tri for any i.  Computed bottom up (the second
// child to arrive at a node computes it); kCollapse then distributes each
// wide node's 8 slots by the same minima.
// ---------------------------------------------------------------------------
constexpr float kCostNode = 1.0f; // a wide-node visit
constexpr float kCostTri  = 1.2f; // a triangle test, relative to a node visit (measured: 0.15-1.2)

__device__ __forceinline__ float halfArea(const float* l, const float* h)
{
    float dx = h[0] - l[0], dy = h[1] - l[1], dz = h[2] - l[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void kDpParents(uint32_t ni, const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                           uint32_t* __restrict__ parent, uint32_t* __restrict__ leafParent)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    uint32_t c[2] = {left[k], right[k]};
    for (int q = 0; q < 2; ++q)
    {
        if (c[q] & kLeafFlag)
            leafParent[c[q] & ~kLeafFlag] = k;
        else
            parent[c[q]] = k;
    }
}

// Slot costs of a child reference: a triangle's for every i, else cost[].
__device__ __forceinline__ void dpRefCosts(uint32_t r, const float* lo, const float* hi, const uint32_t* ids,
                                           const float* cost, float c[8])
{
    if (r & kLeafFlag)
    {
        uint32_t t = ids[r & ~kLeafFlag];
        float    a = halfArea(lo + 3 * size_t(t), hi + 3 * size_t(t)) * kCostTri;
        for (int i = 0; i < 8; ++i) c[i] = a;
    }
    else
        for (int i = 0; i < 8; ++i) c[i] = __ldcg(cost + 8 * size_t(r) + i);
}

__global__ void kDpCosts(uint32_t n, const uint32_t* __restrict__ leafParent, const uint32_t* __restrict__ parent,
                         const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                         const float* __restrict__ lo, const float* __restrict__ hi, const uint32_t* __restrict__ ids,
                         const float* __restrict__ nlo, const float* __restrict__ nhi,
                         const uint32_t* __restrict__ count, float* cost, uint32_t* arrive)
{
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t node = leafParent[j];
    while (node != 0xffffffffu)
    {
        __threadfence();
        if (atomicAdd(&arrive[node], 1u) == 0u) return;
        __threadfence();
        float cl[8], cr[8];
        dpRefCosts(left[node], lo, hi, ids, cost, cl);
        dpRefCosts(right[node], lo, hi, ids, cost, cr);
        float dist[9];
        for (int jj = 2; jj <= 8; ++jj)
        {
            float d = FLT_MAX;
            for (int k = 1; k < jj; ++k) d = fminf(d, cl[k - 1] + cr[jj - k - 1]);
            dist[jj] = d;
        }
        float    A   = halfArea(nlo + 3 * size_t(node), nhi + 3 * size_t(node));
        uint32_t cnt = count[node];
        float    c   = cnt <= 3u ? A * kCostTri * float(cnt) : dist[8] + A * kCostNode;
        float*   out = cost + 8 * size_t(node);
        out[0]       = c;
        for (int i = 2; i <= 8; ++i)
        {
            c          = fminf(c, dist[i]);
            out[i - 1] = c;
        }
        node = parent[node];
    }
}

struct CollapseArgs
{
    const float*    triPos; // 9 floats per triangle, original order
    const float*    lo;     // triangle boxes
    const float*    hi;
    const uint32_t* ids;    // sorted position -> triangle id
    const uint32_t* left;
    const uint32_t* right;
    const float*    nlo;
    const float*    nhi;
    const uint32_t* count;
    const float*    cost; // slot costs of the optimal collapse
    uint4*          nodes;
    float4*         tris;
    uint32_t*       nodeCounter;
    uint32_t*       triCounter;
    uint32_t*       nextCount;
    uint2*          nextTasks;
    float           margin;
    uint32_t        maxNodes;
    uint32_t        maxTris;
    uint32_t*       err;
};

__device__ __forceinline__ uint32_t refCount(const CollapseArgs& A, uint32_t r)
{
    return (r & kLeafFlag) ? 1u : A.count[r];
}

__device__ __forceinline__ uint32_t quantExp(float ext)
{
    // Smallest power of two e with 255 * e >= ext; returns its biased exponent.
    float    x  = ext / 255.0f;
    uint32_t b  = __float_as_uint(x);
    uint32_t ex = (b >> 23) & 0xffu;
    if (b & 0x7fffffu) ex += 1;
    if (ex < 1) ex = 1;
    if (ex > 254) ex = 254;
    float e = __uint_as_float(ex << 23);
    while (e * 255.0f < ext && ex < 254)
    {
        ++ex;
        e = __uint_as_float(ex << 23);
    }
    return ex;
}

// 8-bit planes of a child interval [lo, hi] in the frame (p, e), rounded
// outwards so that the dequantised box p + e * q contains the interval.
__device__ __forceinline__ void quantPlanes(float lo, float hi, float p, float e, uint32_t* ql, uint32_t* qh)
{
    int lo_ = int(floorf((lo - p) / e));
    int hi_ = int(ceilf((hi - p) / e));
    lo_     = max(0, min(255, lo_));
    hi_     = max(0, min(255, hi_));
    while (lo_ > 0 && p + e * float(lo_) > lo) --lo_;
    while (hi_ < 255 && p + e * float(hi_) < hi) ++hi_;
    *ql = uint32_t(lo_);
    *qh = uint32_t(hi_);
}

__global__ void kCollapse(CollapseArgs A, const uint2* __restrict__ tasks, uint32_t ntasks)
{
    uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= ntasks) return;
    uint32_t ref  = tasks[ti].x;
    uint32_t wide = tasks[ti].y;

    uint32_t ch[8];
    int      cnt = 0;
    if ((ref & kLeafFlag) || A.count[ref] <= 3u)
        ch[cnt++] = ref;
    else
    {
        // Distribute the 8 slots by the cost minima: (node, budget) pairs
        // split until a budget of 1 or the cost no longer needs the budget.
        uint32_t sn[16], sj[16];
        int      sp = 0;
        sn[sp]      = ref;
        sj[sp++]    = 8u;
        bool root   = true;
        while (sp > 0 && cnt < 8)
        {
            uint32_t x = sn[--sp], j = sj[sp];
            if (!root && ((x & kLeafFlag) || j == 1u))
            {
                ch[cnt++] = x;
                continue;
            }
            const float* cx = A.cost + 8 * size_t(x);
            uint32_t     i  = j;
            if (!root)
                while (i > 1u && cx[i - 2] == cx[j - 1]) --i; // fewest slots with the same cost
            root = false;
            if (i == 1u)
            {
                ch[cnt++] = x;
                continue;
            }
            float cl[8], cr[8];
            dpRefCosts(A.left[x], A.lo, A.hi, A.ids, A.cost, cl);
            dpRefCosts(A.right[x], A.lo, A.hi, A.ids, A.cost, cr);
            uint32_t bk = 1u;
            float    bc = FLT_MAX;
            for (uint32_t k = 1; k < i; ++k)
            {
                float c = cl[k - 1] + cr[i - k - 1];
                if (c < bc)
                {
                    bc = c;
                    bk = k;
                }
            }
            sn[sp]   = A.right[x];
            sj[sp++] = i - bk;
            sn[sp]   = A.left[x];
            sj[sp++] = bk;
        }
    }

    // Child boxes, parent box (widened by the margin).
    float clo[8][3], chi[8][3], plo[3], phi[3];
    for (int a = 0; a < 3; ++a)
    {
        plo[a] = FLT_MAX;
        phi[a] = -FLT_MAX;
    }
    for (int k = 0; k < cnt; ++k)
    {
        refBox(ch[k], A.lo, A.hi, A.ids, A.nlo, A.nhi, clo[k], chi[k]);
        for (int a = 0; a < 3; ++a)
        {
            clo[k][a] -= A.margin;
            chi[k][a] += A.margin;
            plo[a] = fminf(plo[a], clo[k][a]);
            phi[a] = fmaxf(phi[a], chi[k][a]);
        }
    }

    // Octant slot assignment (greedy on the alignment of child offset and
    // slot direction).
    int   slotOf[8];
    bool  used[8] = {false, false, false, false, false, false, false, false};
    bool  done[8] = {false, false, false, false, false, false, false, false};
    float pc[3];
    for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (plo[a] + phi[a]);
    for (int it = 0; it < cnt; ++it)
    {
        float bestC = -FLT_MAX;
        int   bk = 0, bs = 0;
        for (int k = 0; k < cnt; ++k)
        {
            if (done[k]) continue;
            float dx = 0.5f * (clo[k][0] + chi[k][0]) - pc[0];
            float dy = 0.5f * (clo[k][1] + chi[k][1]) - pc[1];
            float dz = 0.5f * (clo[k][2] + chi[k][2]) - pc[2];
            for (int s = 0; s < 8; ++s)
            {
                if (used[s]) continue;
                float c = ((s & 1) ? dx : -dx) + ((s & 2) ? dy : -dy) + ((s & 4) ? dz : -dz);
                if (c > bestC)
                {
                    bestC = c;
                    bk    = k;
                    bs    = s;
                }
            }
        }
        done[bk]   = true;
        used[bs]   = true;
        slotOf[bk] = bs;
    }
    int childAt[8];
    for (int s = 0; s < 8; ++s) childAt[s] = -1;
    for (int k = 0; k < cnt; ++k) childAt[slotOf[k]] = k;

    uint32_t nInner = 0, nTris = 0;
    for (int k = 0; k < cnt; ++k)
    {
        uint32_t c = refCount(A, ch[k]);
        if (c <= 3u)
            nTris += c;
        else
            ++nInner;
    }
    uint32_t base  = nInner ? atomicAdd(A.nodeCounter, nInner) : 0u;
    uint32_t tbase = atomicAdd(A.triCounter, nTris);
    if (base + nInner > A.maxNodes || tbase + nTris > A.maxTris || wide >= A.maxNodes)
    {
        atomicOr(A.err, 2u);
        return;
    }

    // Quantisation frame.
    uint32_t ex[3];
    float    e[3];
    for (int a = 0; a < 3; ++a)
    {
        ex[a] = quantExp(phi[a] - plo[a]);
        e[a]  = __uint_as_float(ex[a] << 23);
    }
    uint32_t imask = 0, meta[2] = {0, 0}, qlo[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qhi[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    uint32_t innerRank = 0, triOff = 0;
    for (int s = 0; s < 8; ++s)
    {
        int      word = s >> 2, sh = 8 * (s & 3);
        int      k    = childAt[s];
        uint32_t ql[3], qh[3];
        if (k < 0)
        {
            ql[0] = ql[1] = ql[2] = 255u;
            qh[0] = qh[1] = qh[2] = 0u;
        }
        else
        {
            for (int a = 0; a < 3; ++a) quantPlanes(clo[k][a], chi[k][a], plo[a], e[a], &ql[a], &qh[a]);
            uint32_t r = ch[k];
            uint32_t c = refCount(A, r);
            if (c > 3u)
            {
                imask |= 1u << s;
                uint32_t slotIdx        = base + innerRank++;
                uint32_t ti2            = atomicAdd(A.nextCount, 1u);
                A.nextTasks[ti2]        = make_uint2(r, slotIdx);
            }
            else
            {
                // Gather the subtree's triangles (at most 3).
                uint32_t st[4];
                int      sp = 0;
                st[sp++]    = r;
                uint32_t got = 0;
                while (sp > 0)
                {
                    uint32_t x = st[--sp];
                    if (x & kLeafFlag)
                    {
                        uint32_t tid = A.ids[x & ~kLeafFlag];
                        const float* tp = A.triPos + 9 * size_t(tid);
                        float4* dst = A.tris + size_t(tbase + triOff + got) * 3;
                        dst[0]      = make_float4(tp[0], tp[1], tp[2], __uint_as_float(tid));
                        dst[1]      = make_float4(tp[3], tp[4], tp[5], 0.0f);
                        dst[2]      = make_float4(tp[6], tp[7], tp[8], 0.0f);
                        ++got;
                    }
                    else
                    {
                        st[sp++] = A.right[x];
                        st[sp++] = A.left[x];
                    }
                }
                uint32_t unary = (1u << got) - 1u;
                meta[word] |= ((unary << 5) | triOff) << sh;
                triOff += got;
            }
        }
        for (int a = 0; a < 3; ++a)
        {
            qlo[a][word] |= ql[a] << sh;
            qhi[a][word] |= qh[a] << sh;
        }
    }
    uint4* np = A.nodes + size_t(wide) * 5;
    np[0]     = make_uint4(__float_as_uint(plo[0]), __float_as_uint(plo[1]), __float_as_uint(plo[2]),
                           ex[0] | (ex[1] << 8) | (ex[2] << 16) | (imask << 24));
    np[1]     = make_uint4(base, tbase, meta[0], meta[1]);
    np[2]     = make_uint4(qlo[0][0], qlo[0][1], qlo[1][0], qlo[1][1]);
    np[3]     = make_uint4(qlo[2][0], qlo[2][1], qhi[0][0], qhi[0][1]);
    np[4]     = make_uint4(qhi[1][0], qhi[1][1], qhi[2][0], qhi[2][1]);
}

// Validation of a built tree (error bits: 1 exponent outside 1..254, 2 child
// index beyond the node count, 4 leaf triangle range outside the node's 24 or
// the triangle count, 8 triangle ids not a permutation of 0..n-1).
__global__ void kValidateNodes(const uint4* __restrict__ nodes, uint32_t numNodes, uint32_t n, uint32_t* err)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    uint4    n0 = nodes[size_t(i) * 5], n1 = nodes[size_t(i) * 5 + 1];
    uint32_t imask = n0.w >> 24, bits = 0u;
    for (int a = 0; a < 3; ++a)
    {
        uint32_t e = (n0.w >> (8 * a)) & 0xffu;
        if (e < 1u || e > 254u) bits |= 1u;
    }
    if (imask && uint64_t(n1.x) + __popc(imask) > numNodes) bits |= 2u;
    for (int sl = 0; sl < 8; ++sl)
    {
        if (imask & (1u << sl)) continue;
        uint32_t meta = ((sl < 4 ? n1.z : n1.w) >> (8 * (sl & 3))) & 0xffu;
        if (!meta) continue;
        uint32_t off = meta & 31u, unary = meta >> 5;
        uint32_t cnt = unary == 1u ? 1u : unary == 3u ? 2u : unary == 7u ? 3u : 99u;
        if (cnt == 99u || off + cnt > 24u || uint64_t(n1.y) + off + cnt > n) bits |= 4u;
    }
    if (bits) atomicOr(err, bits);
}

__global__ void kValidateTris(const float4* __restrict__ tris, uint32_t n, uint32_t* __restrict__ seen, uint32_t* err)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t id = __float_as_uint(tris[size_t(i) * 3].w);
    if (id >= n)
    {
        atomicOr(err, 8u);
        return;
    }
    uint32_t bit = 1u << (id & 31u);
    if (atomicOr(seen + (id >> 5), bit) & bit) atomicOr(err, 8u);
}

} // namespace

cl_status buildWideBvh(const float* dTri9, uint32_t n, cudaStream_t st, WideBvh* out, std::string* err,
                       BuildArena* arena)
{
    out->release();
    BuildArena  localArena;
    BuildArena& mem = arena ? *arena : localArena;
    mem.reset();
    if (n == 0)
    {
        *err = "cannot build a BVH over zero triangles";
        return CL_ERR_INVALID_ARG;
    }
    ScratchBuf lo, hi, keys, keys2, ids, ids2, left, right, parent, nlo, nhi, count, arrive, bounds, tmp, tasksA, tasksB,
        ctr;
    size_t nn = n;
    CL_TRY(mem.take(lo, nn * 3 * 4, err));
    CL_TRY(mem.take(hi, nn * 3 * 4, err));
    CL_TRY(mem.take(keys, nn * 8, err));
    CL_TRY(mem.take(keys2, nn * 8, err));
    CL_TRY(mem.take(ids, nn * 4, err));
    CL_TRY(mem.take(ids2, nn * 4, err));
    size_t ni = nn > 1 ? nn - 1 : 1;
    CL_TRY(mem.take(left, ni * 4, err));
    CL_TRY(mem.take(right, ni * 4, err));
    CL_TRY(mem.take(parent, (2 * nn) * 4, err));
    CL_TRY(mem.take(nlo, ni * 3 * 4, err));
    CL_TRY(mem.take(nhi, ni * 3 * 4, err));
    CL_TRY(mem.take(count, ni * 4, err));
    CL_TRY(mem.take(arrive, ni * 4, err));
    CL_TRY(mem.take(bounds, sizeof(Bounds), err));
    CL_TRY(mem.take(ctr, 16, err));

    Bounds b0;
    for (int a = 0; a < 3; ++a)
    {
        b0.clo[a] = b0.slo[a] = 0xffffffffu;
        b0.chi[a] = b0.shi[a] = 0u;
    }
    CL_CUDA(cudaMemcpyAsync(bounds.p, &b0, sizeof(b0), cudaMemcpyHostToDevice, st), err);
    uint32_t blocks = (n + 255) / 256;
    kTriBounds<<<blocks, 256, 0, st>>>(dTri9, n, lo.f(), hi.f(), (Bounds*)bounds.p);
    kMorton<<<blocks, 256, 0, st>>>(lo.f(), hi.f(), n, (Bounds*)bounds.p, (uint64_t*)keys.p, ids.u());
    CL_CUDA(cudaGetLastError(), err);

    size_t tmpBytes = 0;
    CL_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, (uint64_t*)keys.p, (uint64_t*)keys2.p, ids.u(), ids2.u(),
                                            int(n), 0, 63, st),
            err);
    CL_TRY(mem.take(tmp, tmpBytes, err));
    CL_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmpBytes, (uint64_t*)keys.p, (uint64_t*)keys2.p, ids.u(), ids2.u(),
                                            int(n), 0, 63, st),
            err);
    tmp.release();
    keys.release();
    ids.release();

    // Binary tree: PLOC over the Morton order (LBVH radix tree as fallback).
    uint32_t rootRef = kLeafFlag; // a single triangle: the root is a leaf
    if (n > 1)
    {
        ScratchBuf C, C2, blo, bhi, blo2, bhi2, nnb, valid, pos, scanTmp;
        CL_TRY(mem.take(C, nn * 4, err));
        CL_TRY(mem.take(C2, nn * 4, err));
        CL_TRY(mem.take(blo, nn * 16, err));
        CL_TRY(mem.take(bhi, nn * 16, err));
        CL_TRY(mem.take(blo2, nn * 16, err));
        CL_TRY(mem.take(bhi2, nn * 16, err));
        CL_TRY(mem.take(nnb, nn * 4, err));
        CL_TRY(mem.take(valid, nn * 4, err));
        CL_TRY(mem.take(pos, nn * 4, err));
        size_t scanBytes = 0;
        CL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, valid.u(), pos.u(), int(n), st), err);
        CL_TRY(mem.take(scanTmp, scanBytes, err));
        CL_CUDA(cudaMemsetAsync(ctr.p, 0, 16, st), err);
        PlocTree T{left.u(), right.u(), nlo.f(), nhi.f(), count.u(), ctr.u()};
        kPlocInit<<<blocks, 256, 0, st>>>(n, ids2.u(), lo.f(), hi.f(), C.u(), blo.as<float4>(), bhi.as<float4>());
        // The cluster count stays on the device (two words, this iteration's
        // and the next's); the host reads it every kPlocCheck iterations to
        // size the launches and to stop.
        constexpr int kPlocCheck = 6;
        ScratchBuf    mbuf;
        CL_TRY(mem.take(mbuf, 8, err));
        CL_CUDA(cudaMemcpyAsync(mbuf.p, &n, 4, cudaMemcpyHostToDevice, st), err);
        uint32_t m = n, iters = 0;
        int      cur = 0;
        while (m > 1 && iters < 4096)
        {
            uint32_t g = (m + kPlocBlock - 1) / kPlocBlock; // m: upper bound of the device count
            for (int k = 0; k < kPlocCheck; ++k)
            {
                const uint32_t* md = mbuf.u() + cur;
                kPlocNearest<<<g, kPlocBlock, 0, st>>>(md, blo.as<float4>(), bhi.as<float4>(), nnb.u());
                kPlocMerge<<<g, kPlocBlock, 0, st>>>(md, m, C.u(), blo.as<float4>(), bhi.as<float4>(), nnb.u(),
                                                     valid.u(), C2.u(), blo2.as<float4>(), bhi2.as<float4>(), T, n - 1);
                CL_CUDA(cub::DeviceScan::ExclusiveSum(scanTmp.p, scanBytes, valid.u(), pos.u(), int(m), st), err);
                kPlocScatter<<<g, kPlocBlock, 0, st>>>(md, valid.u(), pos.u(), C2.u(), blo2.as<float4>(),
                                                       bhi2.as<float4>(), C.u(), blo.as<float4>(), bhi.as<float4>());
                kPlocCount<<<1, 32, 0, st>>>(md, mbuf.u() + (cur ^ 1), valid.u(), pos.u());
                cur ^= 1;
                ++iters;
            }
            CL_CUDA(cudaGetLastError(), err);
            CL_CUDA(cudaMemcpyAsync(&m, mbuf.u() + cur, 4, cudaMemcpyDeviceToHost, st), err);
            CL_CUDA(cudaStreamSynchronize(st), err);
        }
        if (m == 1)
        {
            CL_CUDA(cudaMemcpyAsync(&rootRef, C.p, 4, cudaMemcpyDeviceToHost, st), err);
            CL_CUDA(cudaStreamSynchronize(st), err);
            out->buildIterations = iters;
        }
        else
        {
            // Fall back to the LBVH radix tree (Karras 2012) with bottom-up boxes.
            CL_CUDA(cudaMemsetAsync(parent.p, 0xff, 2 * nn * 4, st), err);
            CL_CUDA(cudaMemsetAsync(arrive.p, 0, ni * 4, st), err);
            kRadixTree<<<(n - 1 + 255) / 256, 256, 0, st>>>((uint64_t*)keys2.p, int(n), left.u(), right.u(),
                                                            parent.u());
            kBottomUp<<<blocks, 256, 0, st>>>(int(n), lo.f(), hi.f(), ids2.u(), left.u(), right.u(), parent.u(),
                                              nlo.f(), nhi.f(), count.u(), arrive.u());
            CL_CUDA(cudaGetLastError(), err);
            rootRef = 0u;
            out->buildIterations = 0;
        }
    }

    Bounds bh;
    CL_CUDA(cudaMemcpyAsync(&bh, bounds.p, sizeof(bh), cudaMemcpyDeviceToHost, st), err);
    CL_CUDA(cudaStreamSynchronize(st), err);
    float margin;
    {
        auto unord = [](uint32_t v) {
            uint32_t bits = (v & 0x80000000u) ? (v & 0x7fffffffu) : ~v;
            float    f;
            memcpy(&f, &bits, 4);
            return f;
        };
        float l[3], h[3];
        for (int a = 0; a < 3; ++a)
        {
            l[a] = unord(bh.slo[a]);
            h[a] = unord(bh.shi[a]);
        }
        margin = sceneMargin(l, h);
    }

    uint32_t maxNodes = n + 1;
    CL_TRY(out->nodes.alloc(size_t(maxNodes) * 80, err));
    CL_TRY(out->tris.alloc(nn * 48, err));
    size_t taskCap = nn / 2 + 8;
    CL_TRY(mem.take(tasksA, taskCap * 8, err));
    CL_TRY(mem.take(tasksB, taskCap * 8, err));
    // ctr: [0] node counter, [1] tri counter, [2] next task count, [3] error
    uint32_t c0[4] = {1u, 0u, 0u, 0u};
    CL_CUDA(cudaMemcpyAsync(ctr.p, c0, 16, cudaMemcpyHostToDevice, st), err);
    uint2 root = make_uint2(rootRef, 0u);
    CL_CUDA(cudaMemcpyAsync(tasksA.p, &root, 8, cudaMemcpyHostToDevice, st), err);

    // Slot costs of the optimal collapse, bottom up over the binary tree.
    ScratchBuf dpCost, dpParent, dpLeafParent;
    if (n > 1)
    {
        CL_TRY(mem.take(dpCost, ni * 8 * 4, err));
        CL_TRY(mem.take(dpParent, ni * 4, err));
        CL_TRY(mem.take(dpLeafParent, nn * 4, err));
        CL_CUDA(cudaMemsetAsync(dpParent.p, 0xff, ni * 4, st), err);
        CL_CUDA(cudaMemsetAsync(dpLeafParent.p, 0xff, nn * 4, st), err);
        CL_CUDA(cudaMemsetAsync(arrive.p, 0, ni * 4, st), err);
        kDpParents<<<uint32_t((ni + 255) / 256), 256, 0, st>>>(uint32_t(n - 1), left.u(), right.u(), dpParent.u(),
                                                               dpLeafParent.u());
        kDpCosts<<<blocks, 256, 0, st>>>(n, dpLeafParent.u(), dpParent.u(), left.u(), right.u(), lo.f(), hi.f(),
                                         ids2.u(), nlo.f(), nhi.f(), count.u(), dpCost.f(), arrive.u());
        CL_CUDA(cudaGetLastError(), err);
    }

    CollapseArgs A;
    A.triPos      = dTri9;
    A.lo          = lo.f();
    A.hi          = hi.f();
    A.ids         = ids2.u();
    A.left        = left.u();
    A.right       = right.u();
    A.nlo         = nlo.f();
    A.nhi         = nhi.f();
    A.count       = count.u();
    A.cost        = n > 1 ? dpCost.f() : nullptr; // n == 1: the root is a leaf
    A.nodes       = (uint4*)out->nodes.p;
    A.tris        = (float4*)out->tris.p;
    A.nodeCounter = ctr.u() + 0;
    A.triCounter  = ctr.u() + 1;
    A.nextCount   = ctr.u() + 2;
    A.margin      = margin;
    A.maxNodes    = maxNodes;
    A.maxTris     = n;
    A.err         = ctr.u() + 3;

    uint32_t ntasks = 1, depth = 0;
    out->levels.assign({0u, 1u});
    ScratchBuf* cur = &tasksA;
    ScratchBuf* nxt = &tasksB;
    while (ntasks > 0)
    {
        ++depth;
        A.nextTasks = (uint2*)nxt->p;
        CL_CUDA(cudaMemsetAsync(ctr.u() + 2, 0, 4, st), err);
        kCollapse<<<(ntasks + 63) / 64, 64, 0, st>>>(A, (const uint2*)cur->p, ntasks);
        CL_CUDA(cudaGetLastError(), err);
        uint32_t hc[4];
        CL_CUDA(cudaMemcpyAsync(hc, ctr.p, 16, cudaMemcpyDeviceToHost, st), err);
        CL_CUDA(cudaStreamSynchronize(st), err);
        if (hc[3])
        {
            *err = "BVH collapse exceeded its node bound";
            return CL_ERR_STATE;
        }
        ntasks = hc[2];
        if (ntasks > taskCap)
        {
            *err = "BVH collapse task list overflow";
            return CL_ERR_STATE;
        }
        std::swap(cur, nxt);
        out->numNodes = hc[0];
        if (hc[0] > out->levels.back()) out->levels.push_back(hc[0]);
        if (hc[1] > n)
        {
            *err = "BVH collapse emitted too many triangles";
            return CL_ERR_STATE;
        }
    }
    out->depth   = depth;
    out->numTris = n;
    // Refit state (24 bytes per node), allocated with the tree so that a
    // refit allocates nothing.
    CL_TRY(out->exact.alloc(size_t(out->numNodes) * 24, err));
    CL_TRY(out->scene.alloc(64, err));
    // Validation of every index the traversal kernels will follow, on the
    // device; one error word comes back.
    {
        ScratchBuf verr, seen;
        CL_TRY(mem.take(verr, 4, err));
        CL_TRY(mem.take(seen, (size_t(n) + 31) / 32 * 4, err));
        CL_CUDA(cudaMemsetAsync(verr.p, 0, 4, st), err);
        CL_CUDA(cudaMemsetAsync(seen.p, 0, (size_t(n) + 31) / 32 * 4, st), err);
        kValidateNodes<<<(out->numNodes + 255) / 256, 256, 0, st>>>(out->nodes.as<const uint4>(), out->numNodes, n,
                                                                       verr.u());
        kValidateTris<<<(n + 255) / 256, 256, 0, st>>>(out->tris.as<const float4>(), n, seen.u(), verr.u());
        CL_CUDA(cudaGetLastError(), err);
        uint32_t bad = 0;
        CL_CUDA(cudaMemcpyAsync(&bad, verr.p, 4, cudaMemcpyDeviceToHost, st), err);
        CL_CUDA(cudaStreamSynchronize(st), err);
        if (bad)
        {
            *err = (bad & 1u)   ? "BVH validation: bad exponent"
                   : (bad & 2u) ? "BVH validation: child index out of range"
                   : (bad & 4u) ? "BVH validation: leaf triangle range out of bounds"
                                : "BVH validation: triangle ids are not a permutation";
            return CL_ERR_STATE;
        }
    }
    if (depth + 1 > uint32_t(kStackDepth))
    {
        *err = "BVH depth " + std::to_string(depth) + " exceeds the traversal stack";
        return CL_ERR_STATE;
    }
    return CL_OK;
}

namespace
{
constexpr int kRefitBlock = 128;

// Leaf triangles from the vertex array; scene bounds into bounds[0..5] as
// ordered ints (min x,y,z then max x,y,z): grid-stride, reduced per block,
// one atomic per block and value.
__global__ void __launch_bounds__(256) kRefitTris(float4* __restrict__ tris, uint32_t n, const float4* __restrict__ vtx,
                                                  const uint4* __restrict__ triIdx, uint32_t* __restrict__ bounds)
{
    __shared__ uint32_t part[6][8];
    uint32_t            ol[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, oh[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float4*  t   = tris + 3 * size_t(i);
        uint32_t tid = __float_as_uint(t[0].w);
        uint4    ix  = triIdx[tid];
        float4   a = vtx[3 * size_t(ix.x)], b = vtx[3 * size_t(ix.y)], c = vtx[3 * size_t(ix.z)];
        t[0]         = make_float4(a.x, a.y, a.z, __uint_as_float(tid));
        t[1]         = make_float4(b.x, b.y, b.z, 0.0f);
        t[2]         = make_float4(c.x, c.y, c.z, 0.0f);
        float l[3] = {fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z)};
        float h[3] = {fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z)};
        for (int k = 0; k < 3; ++k)
        {
            ol[k] = min(ol[k], fordered(l[k]));
            oh[k] = max(oh[k], fordered(h[k]));
        }
    }
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1)
        {
            ol[k] = min(ol[k], __shfl_xor_sync(0xffffffffu, ol[k], o));
            oh[k] = max(oh[k], __shfl_xor_sync(0xffffffffu, oh[k], o));
        }
    if (lane == 0)
        for (int k = 0; k < 3; ++k)
        {
            part[k][warp]     = ol[k];
            part[3 + k][warp] = oh[k];
        }
    __syncthreads();
    if (threadIdx.x < 6)
    {
        int      k = threadIdx.x;
        uint32_t v = part[k][0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) v = k < 3 ? min(v, part[k][w]) : max(v, part[k][w]);
        if (k < 3)
        {
            if (v != 0xffffffffu) atomicMin(bounds + k, v);
        }
        else if (v != 0u)
            atomicMax(bounds + k, v);
    }
}

// One tree level, eight lanes per node (lane s = child slot s): each lane
// boxes its slot (the child's exact box from the level below, or its leaf
// triangles), the group reduces the node's exact and widened boxes, every
// lane quantises its own slot in the node's frame, and lane 0 writes the
// node.  Topology (imask, child and triangle bases, leaf metadata, slot
// order) is kept; the result equals kCollapse's for unchanged triangles.
__global__ void __launch_bounds__(128) kRefitLevel(uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                   float* __restrict__ exact, uint32_t first, uint32_t count,
                                                   const uint32_t* __restrict__ bounds)
{
    uint32_t g     = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t t     = g >> 3;
    int      s     = int(g & 7u);
    bool     valid = t < count;
    uint32_t node  = first + (valid ? t : 0u);
    float    sl[3], sh[3];
    for (int a = 0; a < 3; ++a)
    {
        sl[a] = funordered(bounds[a]);
        sh[a] = funordered(bounds[3 + a]);
    }
    float  margin = sceneMargin(sl, sh);
    uint4* np     = nodes + size_t(node) * 5;
    uint4  n0 = make_uint4(0, 0, 0, 0), n1 = make_uint4(0, 0, 0, 0);
    if (valid)
    {
        n0 = np[0];
        n1 = np[1];
    }
    uint32_t imask = n0.w >> 24;
    float    lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    bool     present = false;
    if (valid)
    {
        if (imask & (1u << s))
        {
            uint32_t     c = n1.x + __popc(imask & ((1u << s) - 1u));
            const float* x = exact + 6 * size_t(c);
            for (int a = 0; a < 3; ++a)
            {
                lo[a] = x[a];
                hi[a] = x[3 + a];
            }
            present = true;
        }
        else
        {
            uint32_t m = ((s < 4 ? n1.z : n1.w) >> (8 * (s & 3))) & 0xffu;
            if (m)
            {
                uint32_t off = m & 31u, cnt = __popc(m >> 5);
                for (uint32_t j = 0; j < cnt; ++j)
                {
                    const float4* tp = tris + size_t(n1.y + off + j) * 3;
                    for (int v = 0; v < 3; ++v)
                    {
                        float4 p = tp[v];
                        lo[0] = fminf(lo[0], p.x);
                        lo[1] = fminf(lo[1], p.y);
                        lo[2] = fminf(lo[2], p.z);
                        hi[0] = fmaxf(hi[0], p.x);
                        hi[1] = fmaxf(hi[1], p.y);
                        hi[2] = fmaxf(hi[2], p.z);
                    }
                }
                present = true;
            }
        }
    }
    // Exact box of the node and its widened frame box (group of 8 lanes).
    float xlo[3], xhi[3], clo[3], chi[3], plo[3], phi[3];
    for (int a = 0; a < 3; ++a)
    {
        xlo[a] = lo[a];
        xhi[a] = hi[a];
        clo[a] = present ? lo[a] - margin : FLT_MAX;
        chi[a] = present ? hi[a] + margin : -FLT_MAX;
        plo[a] = clo[a];
        phi[a] = chi[a];
        for (int o = 1; o < 8; o <<= 1)
        {
            xlo[a] = fminf(xlo[a], __shfl_xor_sync(0xffffffffu, xlo[a], o, 8));
            xhi[a] = fmaxf(xhi[a], __shfl_xor_sync(0xffffffffu, xhi[a], o, 8));
            plo[a] = fminf(plo[a], __shfl_xor_sync(0xffffffffu, plo[a], o, 8));
            phi[a] = fmaxf(phi[a], __shfl_xor_sync(0xffffffffu, phi[a], o, 8));
        }
    }
    uint32_t ex[3], ql[3] = {255u, 255u, 255u}, qh[3] = {0u, 0u, 0u};
    for (int a = 0; a < 3; ++a)
    {
        ex[a] = quantExp(phi[a] - plo[a]);
        if (present) quantPlanes(clo[a], chi[a], plo[a], __uint_as_float(ex[a] << 23), &ql[a], &qh[a]);
    }
    // Pack the slot bytes: OR within each quad of lanes, then bring the
    // second quad's words to lane 0.
    uint32_t wl[3], wh[3];
    for (int a = 0; a < 3; ++a)
    {
        wl[a] = ql[a] << (8 * (s & 3));
        wh[a] = qh[a] << (8 * (s & 3));
        for (int o = 1; o < 4; o <<= 1)
        {
            wl[a] |= __shfl_xor_sync(0xffffffffu, wl[a], o, 8);
            wh[a] |= __shfl_xor_sync(0xffffffffu, wh[a], o, 8);
        }
    }
    uint32_t wl1[3], wh1[3];
    for (int a = 0; a < 3; ++a)
    {
        wl1[a] = __shfl_down_sync(0xffffffffu, wl[a], 4, 8);
        wh1[a] = __shfl_down_sync(0xffffffffu, wh[a], 4, 8);
    }
    if (valid && s == 0)
    {
        np[0] = make_uint4(__float_as_uint(plo[0]), __float_as_uint(plo[1]), __float_as_uint(plo[2]),
                           ex[0] | (ex[1] << 8) | (ex[2] << 16) | (imask << 24));
        np[2] = make_uint4(wl[0], wl1[0], wl[1], wl1[1]);
        np[3] = make_uint4(wl[2], wl1[2], wh[0], wh1[0]);
        np[4] = make_uint4(wh[1], wh1[1], wh[2], wh1[2]);
        float* x = exact + 6 * size_t(node);
        for (int a = 0; a < 3; ++a)
        {
            x[a]     = xlo[a];
            x[3 + a] = xhi[a];
        }
    }
}

__device__ __forceinline__ double boxArea(float lx, float ly, float lz, float hx, float hy, float hz)
{
    double dx = double(hx) - lx, dy = double(hy) - ly, dz = double(hz) - lz;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

// Sum over all child slots of (dequantised box area) x (1 for an inner
// child, its triangle count for a leaf), into *sum.
__global__ void kSahSum(const uint4* __restrict__ nodes, uint32_t n, double* sum)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double   c = 0.0;
    if (i < n)
    {
        const uint4* np = nodes + size_t(i) * 5;
        uint4        n0 = np[0], n1 = np[1], n2 = np[2], n3 = np[3], n4 = np[4];
        float        px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
        float        ex = __uint_as_float((n0.w & 0xffu) << 23), ey = __uint_as_float(((n0.w >> 8) & 0xffu) << 23),
              ez = __uint_as_float(((n0.w >> 16) & 0xffu) << 23);
        uint32_t imask = n0.w >> 24;
        for (int s = 0; s < 8; ++s)
        {
            int      w = s >> 2, sh = 8 * (s & 3);
            uint32_t lx = ((w ? n2.y : n2.x) >> sh) & 0xffu, ly = ((w ? n2.w : n2.z) >> sh) & 0xffu,
                     lz = ((w ? n3.y : n3.x) >> sh) & 0xffu;
            uint32_t hx = ((w ? n3.w : n3.z) >> sh) & 0xffu, hy = ((w ? n4.y : n4.x) >> sh) & 0xffu,
                     hz = ((w ? n4.w : n4.z) >> sh) & 0xffu;
            if (lx > hx) continue; // empty slot
            double weight;
            if (imask & (1u << s))
                weight = 1.0;
            else
            {
                uint32_t m = ((w ? n1.w : n1.z) >> sh) & 0xffu;
                weight     = double(__popc(m >> 5));
            }
            c += weight * boxArea(px + ex * float(lx), py + ey * float(ly), pz + ez * float(lz), px + ex * float(hx),
                                  py + ey * float(hy), pz + ez * float(hz));
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c != 0.0) atomicAdd(sum, c);
}

__global__ void kGatherTri9(const float4* __restrict__ vtx, const uint4* __restrict__ triIdx, uint32_t n,
                            float* __restrict__ tri9)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 ix = triIdx[i];
    float4 a = vtx[3 * size_t(ix.x)], b = vtx[3 * size_t(ix.y)], c = vtx[3 * size_t(ix.z)];
    float* o = tri9 + 9 * size_t(i);
    o[0] = a.x; o[1] = a.y; o[2] = a.z;
    o[3] = b.x; o[4] = b.y; o[5] = b.z;
    o[6] = c.x; o[7] = c.y; o[8] = c.z;
}
} // namespace

cl_status refitWideBvh(WideBvh* bvh, const void* vtx, const void* triIdx, cudaStream_t st, std::string* err)
{
    if (!bvh->nodes.p || bvh->levels.size() < 2 || bvh->levels.back() != bvh->numNodes)
    {
        *err = "refit needs a built BVH";
        return CL_ERR_STATE;
    }
    if (bvh->exact.bytes < size_t(bvh->numNodes) * 24 || !bvh->scene.p)
    {
        *err = "refit buffers missing";
        return CL_ERR_STATE;
    }
    // Bounds start at (+inf ordered, -inf ordered): 0xff bytes for the
    // minima, zero bytes for the maxima.
    CL_CUDA(cudaMemsetAsync(bvh->scene.p, 0xff, 12, st), err);
    CL_CUDA(cudaMemsetAsync(bvh->scene.u() + 3, 0, 12, st), err);
    uint32_t n = bvh->numTris;
    static int sms = 0;
    if (!sms)
    {
        int dev = 0;
        CL_CUDA(cudaGetDevice(&dev), err);
        CL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), err);
    }
    uint32_t blocks = std::min<uint32_t>((n + 255) / 256, uint32_t(sms) * 8u);
    kRefitTris<<<blocks, 256, 0, st>>>(bvh->tris.as<float4>(), n, static_cast<const float4*>(vtx),
                                       static_cast<const uint4*>(triIdx), bvh->scene.u());
    CL_CUDA(cudaGetLastError(), err);
    for (size_t d = bvh->levels.size() - 1; d-- > 0;)
    {
        uint32_t first = bvh->levels[d], count = bvh->levels[d + 1] - first;
        uint64_t lanes = uint64_t(count) * 8u;
        kRefitLevel<<<uint32_t((lanes + kRefitBlock - 1) / kRefitBlock), kRefitBlock, 0, st>>>(
            bvh->nodes.as<uint4>(), bvh->tris.as<const float4>(), bvh->exact.f(), first, count, bvh->scene.u());
        CL_CUDA(cudaGetLastError(), err);
    }
    return CL_OK;
}

cl_status wideBvhSahCost(WideBvh& bvh, cudaStream_t st, double* cost, std::string* err)
{
    if (!bvh.nodes.p || bvh.numNodes == 0)
    {
        *err = "no BVH";
        return CL_ERR_STATE;
    }
    if (!bvh.scene.p) CL_TRY(bvh.scene.alloc(64, err));
    double* sum = reinterpret_cast<double*>(bvh.scene.as<char>() + 32);
    CL_CUDA(cudaMemsetAsync(sum, 0, 8, st), err);
    kSahSum<<<(bvh.numNodes + 255) / 256, 256, 0, st>>>(bvh.nodes.as<const uint4>(), bvh.numNodes, sum);
    CL_CUDA(cudaGetLastError(), err);
    double                total = 0.0;
    std::vector<uint32_t> h(20);
    CL_CUDA(cudaMemcpyAsync(&total, sum, 8, cudaMemcpyDeviceToHost, st), err);
    CL_CUDA(cudaMemcpyAsync(h.data(), bvh.nodes.p, 80, cudaMemcpyDeviceToHost, st), err);
    CL_CUDA(cudaStreamSynchronize(st), err);
    // Root box extent per axis: e * (largest qhi - smallest qlo) over the
    // root's present slots (qlo words at h[8 + 2a + w], qhi at h[14 + 2a + w]).
    double ext[3];
    for (int a = 0; a < 3; ++a)
    {
        uint32_t eb = ((h[3] >> (8 * a)) & 0xffu) << 23;
        float    e;
        memcpy(&e, &eb, 4);
        uint32_t qlo = 255, qhi = 0;
        for (int sl = 0; sl < 8; ++sl)
        {
            int      w = sl >> 2, sh = 8 * (sl & 3);
            uint32_t lo = (h[8 + 2 * a + w] >> sh) & 0xffu, hi = (h[14 + 2 * a + w] >> sh) & 0xffu;
            if (lo > hi) continue;
            qlo = std::min(qlo, lo);
            qhi = std::max(qhi, hi);
        }
        ext[a] = qhi >= qlo ? double(e) * double(qhi - qlo) : 0.0;
    }
    double rootArea = 2.0 * (ext[0] * ext[1] + ext[1] * ext[2] + ext[2] * ext[0]);
    *cost           = rootArea > 0.0 ? 1.0 + total / rootArea : 0.0;
    return CL_OK;
}

cl_status gatherTrianglePositions(const void* vtx, const void* triIdx, uint32_t n, float* tri9, cudaStream_t st,
                                  std::string* err)
{
    kGatherTri9<<<(n + 255) / 256, 256, 0, st>>>(static_cast<const float4*>(vtx), static_cast<const uint4*>(triIdx),
                                                  n, tri9);
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

} // namespace clb
