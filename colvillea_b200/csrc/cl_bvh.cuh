// 8-wide compressed BVH: node layout and traversal (closest hit / any hit).
//
// Replaces OptiX's acceleration structures and optixTrace
// (src/core/devices/optixdevice.cpp:136-233, src/core/devices/optix.cu:38-110):
// B200 has no RT cores, so traversal runs on the SMs.
//
// Node (80 bytes = 5 x uint4), after the compressed wide BVH of Ylitie,
// Karras and Laine (HPG 2017):
//   n0 = {p.x, p.y, p.z, ex | ey<<8 | ez<<16 | imask<<24}
//   n1 = {childBase, triBase, meta[0..3], meta[4..7]}
//   n2 = {qlo.x[0..3], qlo.x[4..7], qlo.y[0..3], qlo.y[4..7]}
//   n3 = {qlo.z[0..3], qlo.z[4..7], qhi.x[0..3], qhi.x[4..7]}
//   n4 = {qhi.y[0..3], qhi.y[4..7], qhi.z[0..3], qhi.z[4..7]}
// Child box of slot s: p + 2^(e-127) * q.  imask bit s: slot s is an inner
// node, stored at childBase + popc(imask & ((1<<s)-1)).  Leaf slot meta:
// (unary triangle count << 5) | offset from triBase (at most 3 triangles per
// leaf, 24 per node).  Empty slots have qlo = 255, qhi = 0 (never hit).
// Slots are assigned by octant: slot bit a set means the child lies on the +a
// side of its parent, so visiting keys (slot ^ ray-octant) in increasing order
// is roughly front to back.
//
// Triangles: 3 float4 per triangle in leaf order {v0.xyz, prim id bits},
// {v1.xyz, 0}, {v2.xyz, 0}.
#pragma once

#include "cl_device.cuh"

namespace clb
{
constexpr int kStackDepth    = 24; // bound checked against the built tree depth
constexpr int kTraceBlock    = 128;
constexpr uint32_t kMissPrim = 0xffffffffu;

struct BvhView
{
    const uint4* __restrict__ nodes;
    const float4* __restrict__ tris;
};

struct TraceCounters
{
    uint32_t nodes, tris;
};

// Exact float of byte b of `word`: PRMT builds 0x4B0000bb (= 2^23 + byte as
// a float) and one FADD removes 2^23; both run on full-rate pipes (an I2F
// conversion would go through the quarter-rate XU pipe).
__device__ __forceinline__ float byteAt(uint32_t word, int b)
{
    return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7440u | uint32_t(b))) - 8388608.0f;
}

// Intersects the ray with the 8 children of one node; returns the hit mask:
// bits 24..31 inner-child keys (slot ^ octant), bits 0..23 triangle offsets.
__device__ __forceinline__ uint32_t intersectNode(const BvhView& bvh, uint32_t idx, f3 o, f3 inv, uint32_t oct, float tmin,
                                                  float tmax, uint32_t* childBase, uint32_t* triBase, uint32_t* imaskOut)
{
    const uint4* np = bvh.nodes + size_t(idx) * 5;
    uint4        n0 = __ldg(np + 0);
    uint4        n1 = __ldg(np + 1);
    uint4        n2 = __ldg(np + 2);
    uint4        n3 = __ldg(np + 3);
    uint4        n4 = __ldg(np + 4);
    float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    float sx = __uint_as_float((n0.w & 0xffu) << 23);
    float sy = __uint_as_float(((n0.w >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23);
    uint32_t imask = n0.w >> 24;
    *childBase     = n1.x;
    *triBase       = n1.y;
    *imaskOut      = imask;
    float idx_ = sx * inv.x, idy = sy * inv.y, idz = sz * inv.z;
    float ox = (px - o.x) * inv.x, oy = (py - o.y) * inv.y, oz = (pz - o.z) * inv.z;
    // Near/far quantised planes per axis, by ray direction sign.
    bool     nx = inv.x < 0.0f, ny = inv.y < 0.0f, nz = inv.z < 0.0f;
    uint32_t loxA = nx ? n3.z : n2.x, loxB = nx ? n3.w : n2.y, hixA = nx ? n2.x : n3.z, hixB = nx ? n2.y : n3.w;
    uint32_t loyA = ny ? n4.x : n2.z, loyB = ny ? n4.y : n2.w, hiyA = ny ? n2.z : n4.x, hiyB = ny ? n2.w : n4.y;
    uint32_t lozA = nz ? n4.z : n3.x, lozB = nz ? n4.w : n3.y, hizA = nz ? n3.x : n4.z, hizB = nz ? n3.y : n4.w;
    uint32_t hits = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s)
    {
        const int b   = s & 3;
        uint32_t  lx  = s < 4 ? loxA : loxB, hx = s < 4 ? hixA : hixB;
        uint32_t  ly  = s < 4 ? loyA : loyB, hy = s < 4 ? hiyA : hiyB;
        uint32_t  lz  = s < 4 ? lozA : lozB, hz = s < 4 ? hizA : hizB;
        float tnx = __fmaf_rn(byteAt(lx, b), idx_, ox), tfx = __fmaf_rn(byteAt(hx, b), idx_, ox);
        float tny = __fmaf_rn(byteAt(ly, b), idy, oy), tfy = __fmaf_rn(byteAt(hy, b), idy, oy);
        float tnz = __fmaf_rn(byteAt(lz, b), idz, oz), tfz = __fmaf_rn(byteAt(hz, b), idz, oz);
        float tn  = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
        float tf  = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
        if (tn <= tf)
        {
            if (imask & (1u << s))
                hits |= 1u << (24 + (s ^ oct));
            else
            {
                uint32_t meta = (s < 4 ? n1.z : n1.w) >> (8 * b) & 0xffu;
                hits |= (meta >> 5) << (meta & 31u);
            }
        }
    }
    return hits;
}

// Per-ray traversal state, advanced one node (plus that node's triangles) per
// step so that a warp can refill lanes whose ray finished.
struct Trav
{
    RayPre   pre;
    f3       inv;
    uint32_t oct;
    float    tmin, tmax;
    uint2    ng, tg;
    int      sp;
    uint32_t best;
    float    bt, b1, b2;
};

__device__ __forceinline__ void travInit(Trav& s, f3 o, f3 d, float tmin, float tmax)
{
    s.pre   = rayPrepare(o, d);
    s.inv.x = 1.0f / (fabsf(d.x) < 1e-30f ? copysignf(1e-30f, d.x) : d.x);
    s.inv.y = 1.0f / (fabsf(d.y) < 1e-30f ? copysignf(1e-30f, d.y) : d.y);
    s.inv.z = 1.0f / (fabsf(d.z) < 1e-30f ? copysignf(1e-30f, d.z) : d.z);
    s.oct   = (s.inv.x < 0.0f ? 1u : 0u) | (s.inv.y < 0.0f ? 2u : 0u) | (s.inv.z < 0.0f ? 4u : 0u);
    s.tmin  = tmin;
    s.tmax  = tmax;
    // The root is slot 0 of a virtual parent: key = oct, imask = 1.
    s.ng   = make_uint2(0u, (1u << (24 + s.oct)) | 1u);
    s.tg   = make_uint2(0u, 0u);
    s.sp   = 0;
    s.best = kMissPrim;
    s.bt   = tmax;
    s.b1 = s.b2 = 0.0f;
}

// One traversal step.  ANY: stop at the first hit in (tmin, tmax) (shadow
// rays; the reference searches for the closest hit there, optix.cu:99-109,
// which gives the same visibility).  Closest: smallest t in (tmin, tmax),
// ties to the lower primitive id.  `stack` points at this thread's column of
// a shared [kStackDepth][kTraceBlock] array.  Returns true when the ray is
// finished (s.best: primitive id or kMissPrim; s.bt, s.b1, s.b2).
template <bool ANY, bool STATS>
__device__ __forceinline__ bool travStep(const BvhView& bvh, Trav& s, uint2* stack, TraceCounters* cnt, uint32_t* err)
{
    if (s.ng.y > 0x00ffffffu)
    {
        uint32_t key = __ffs(s.ng.y >> 24) - 1;
        s.ng.y &= ~(1u << (24 + key));
        uint32_t slot  = key ^ s.oct;
        uint32_t imask = s.ng.y & 0xffu;
        uint32_t child = s.ng.x + __popc(imask & ((1u << slot) - 1u));
        if (s.ng.y > 0x00ffffffu)
        {
            if (s.sp >= kStackDepth)
            {
                atomicOr(err, 1u);
                s.best = kMissPrim;
                return true;
            }
            stack[s.sp * kTraceBlock] = s.ng;
            ++s.sp;
        }
        uint32_t cb, tb, im;
        uint32_t hits = intersectNode(bvh, child, s.pre.o, s.inv, s.oct, s.tmin, s.bt, &cb, &tb, &im);
        if (STATS) cnt->nodes++;
        s.ng = make_uint2(cb, (hits & 0xff000000u) | im);
        s.tg = make_uint2(tb, hits & 0x00ffffffu);
    }
    while (s.tg.y)
    {
        uint32_t k = __ffs(s.tg.y) - 1;
        s.tg.y &= ~(1u << k);
        const float4* tp = bvh.tris + size_t(s.tg.x + k) * 3;
        float4        a  = __ldg(tp + 0);
        float4        b  = __ldg(tp + 1);
        float4        c  = __ldg(tp + 2);
        if (STATS) cnt->tris++;
        float t, u, v;
        if (intersectTri(s.pre, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, f3{c.x, c.y, c.z}, &t, &u, &v) && t > s.tmin)
        {
            uint32_t id = __float_as_uint(a.w);
            if (ANY)
            {
                if (t < s.tmax)
                {
                    s.bt   = t;
                    s.best = id;
                    return true;
                }
            }
            else if (t < s.bt || (t == s.bt && id < s.best))
            {
                s.bt   = t;
                s.best = id;
                s.b1   = u;
                s.b2   = v;
            }
        }
    }
    if (s.ng.y <= 0x00ffffffu)
    {
        if (s.sp == 0) return true;
        --s.sp;
        s.ng = stack[s.sp * kTraceBlock];
    }
    return false;
}

// Whole traversal of one ray (used where lanes are not refilled).
template <bool ANY, bool STATS>
__device__ __forceinline__ uint32_t traverse(const BvhView& bvh, f3 o, f3 d, float tmin, float tmax, float* tHit,
                                             float* b1Hit, float* b2Hit, uint2* stack, TraceCounters* cnt,
                                             uint32_t* err)
{
    Trav s;
    travInit(s, o, d, tmin, tmax);
    while (!travStep<ANY, STATS>(bvh, s, stack, cnt, err))
    {
    }
    *tHit  = s.bt;
    *b1Hit = s.b1;
    *b2Hit = s.b2;
    return s.best;
}

} // namespace clb
