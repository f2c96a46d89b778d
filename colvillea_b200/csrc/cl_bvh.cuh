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
// Leaf triangles tested per traversal step.  A node's triangles are tested
// one per step and the next node is visited only after them, so the visit
// order is unchanged; but a lane with a long leaf no longer holds its warp in
// a loop while the other lanes wait: they take their own node steps meanwhile
// (1 was faster than 2, 4, 8 or all at once on configs 2 and 5).
constexpr int kTrisPerStep = 1;
constexpr int kTraceBlock    = 128;
constexpr uint32_t kMissPrim = 0xffffffffu;

// Two-level scenes (CL_TWO_LEVEL): one tree per mesh in object space, and a
// top tree over the instances' world boxes whose leaf entries are instances
// (the w of a top-tree triangle record holds the instance index).  A ray that
// reaches an instance entry continues in that mesh's tree with the ray mapped
// to object space (same parameter t: the map is affine).
struct InstDev
{
    float4        w2o[3];   // object-from-world rows {m0, m1, m2, translation}
    float4        o2w[3];   // world-from-object rows
    const uint4*  nodes;    // the mesh's tree
    const float4* tris;
    uint32_t      primBase; // global id of the instance's first triangle (instance order)
    uint32_t      triBase;  // the mesh's first entry in the triangle index pool
    uint32_t      material;
    uint32_t      flags;    // bit 0: the transform mirrors (negative determinant)
};

struct BvhView
{
    const uint4* __restrict__ nodes;
    const float4* __restrict__ tris;
    const InstDev* __restrict__ inst; // two-level: the instances (nodes/tris are the top tree); null otherwise
    // Traversal stack entries per thread: the tree's depth + 1 (a ray holds
    // at most one pending node group per level), at most kStackDepth.  The
    // kernels' dynamic shared memory is stackDepth * kTraceBlock * 8 bytes,
    // so that a shallow tree leaves more of the SM's on-chip memory to L1.
    uint32_t stackDepth;
};

// Lane refill in the persistent traversal kernels of flattened scenes: a lane
// runs up to kRefillSteps traversal steps with no warp-synchronous operation
// (a vote in every step would make the warp reconverge at each step, which
// cost more than the idle lanes it saves), then the warp votes and, when at
// least kRefillIdle lanes are idle, gives them the next rays.  Measured on
// config 2 (1920x1080, 4.7 M triangles): 2-6 idle lanes and 3-6 steps are
// within 1% of each other; 1 step (a vote per step) was 60% slower than no
// refill at all, 16 steps 4% slower than 4.
constexpr uint32_t kRefillIdle  = 4;
constexpr uint32_t kRefillSteps = 4;

__host__ __device__ constexpr size_t traceStackBytes(uint32_t depth) { return size_t(depth) * kTraceBlock * 8u; }

struct TraceCounters
{
    uint32_t nodes, tris;
};

// Quantised planes are decoded exactly without a conversion instruction:
// PRMT builds 0x4B0000bb (= 2^23 + byte as a float) and a subtraction of
// 2^23 leaves the byte (an I2F would go through the quarter-rate XU pipe).
// Byte b of wa and of wb as 2^23 + byte (floats), for the paired plane math.
__device__ __forceinline__ float2 bytePair(uint32_t wa, uint32_t wb, int b)
{
    return make_float2(__uint_as_float(__byte_perm(wa, 0x4B000000u, 0x7440u | uint32_t(b))),
                       __uint_as_float(__byte_perm(wb, 0x4B000000u, 0x7440u | uint32_t(b))));
}

// Three-input minimum and maximum (sm_100 min.f32 / max.f32 with three
// operands; exact, like the nested two-input forms).
__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Child-key table (shared memory, kKeyLutBytes per block): entry oct * 256 + m
// is the 8-bit slot mask m with each slot s moved to bit s ^ oct, the order in
// which a ray of octant oct visits the children.  One table lookup per node
// replaces three conditional bit swaps on the busiest (integer) pipe.
constexpr int kKeyLutBytes = 8 * 256;
__device__ __forceinline__ void fillKeyLut(uint8_t* lut)
{
    for (int i = threadIdx.x; i < kKeyLutBytes; i += blockDim.x)
    {
        uint32_t oct = uint32_t(i) >> 8, k = uint32_t(i) & 0xffu;
        k = (oct & 1u) ? (((k & 0x55u) << 1) | ((k >> 1) & 0x55u)) : k;
        k = (oct & 2u) ? (((k & 0x33u) << 2) | ((k >> 2) & 0x33u)) : k;
        k = (oct & 4u) ? (((k & 0x0fu) << 4) | ((k >> 4) & 0x0fu)) : k;
        lut[i] = uint8_t(k);
    }
    __syncthreads();
}

// Intersects the ray with the 8 children of one node; returns the hit mask:
// bits 24..31 inner-child keys (slot ^ octant), bits 0..23 triangle offsets.
__device__ __forceinline__ uint32_t intersectNode(const uint4* __restrict__ nodes, uint32_t idx, f3 o, f3 inv, uint32_t oct,
                                                  float tmin, float tmax, uint32_t* childBase, uint32_t* triBase,
                                                  uint32_t* imaskOut, const uint8_t* keyLut)
{
    const uint4* np = nodes + size_t(idx) * 5;
    const uint4  n0 = __ldg(np + 0), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
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
    // Slots b and b + 4 as one float2 pair: 2^23 + byte from PRMT, exact
    // byte by FADD2, plane distance by FFMA2 (each lane IEEE round to
    // nearest, so the values equal the scalar fmaf(q, scale, offset)); the
    // slab interval by 3-input min/max.
    const float2 bias = make_float2(-8388608.0f, -8388608.0f);
    const float2 sX = make_float2(idx_, idx_), sY = make_float2(idy, idy), sZ = make_float2(idz, idz);
    const float2 oX = make_float2(ox, ox), oY = make_float2(oy, oy), oZ = make_float2(oz, oz);
    uint32_t     hitSlots = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
    {
        float2 tnx = __ffma2_rn(__fadd2_rn(bytePair(loxA, loxB, b), bias), sX, oX);
        float2 tfx = __ffma2_rn(__fadd2_rn(bytePair(hixA, hixB, b), bias), sX, oX);
        float2 tny = __ffma2_rn(__fadd2_rn(bytePair(loyA, loyB, b), bias), sY, oY);
        float2 tfy = __ffma2_rn(__fadd2_rn(bytePair(hiyA, hiyB, b), bias), sY, oY);
        float2 tnz = __ffma2_rn(__fadd2_rn(bytePair(lozA, lozB, b), bias), sZ, oZ);
        float2 tfz = __ffma2_rn(__fadd2_rn(bytePair(hizA, hizB, b), bias), sZ, oZ);
        float  tn0 = max3f(tnx.x, tny.x, fmaxf(tnz.x, tmin)), tf0 = min3f(tfx.x, tfy.x, fminf(tfz.x, tmax));
        float  tn1 = max3f(tnx.y, tny.y, fmaxf(tnz.y, tmin)), tf1 = min3f(tfx.y, tfy.y, fminf(tfz.y, tmax));
        hitSlots |= (tn0 <= tf0 ? 1u << b : 0u) | (tn1 <= tf1 ? 1u << (b + 4) : 0u);
    }
    // Inner children: slot s -> key s ^ oct (bit permutation of the mask, from the table).
    uint32_t hits = uint32_t(keyLut[(oct << 8) | (hitSlots & imask)]) << 24;
    // Leaf children: their triangle ranges (unary count << 5 | offset).
    uint32_t leaf = hitSlots & ~imask;
    while (leaf)
    {
        uint32_t sl   = __ffs(leaf) - 1;
        leaf &= leaf - 1u;
        uint32_t meta = ((sl < 4 ? n1.z : n1.w) >> (8 * (sl & 3u))) & 0xffu;
        hits |= (meta >> 5) << (meta & 31u);
    }
    return hits;
}

// Per-ray traversal state, advanced one step at a time: a node test (when no
// triangle of the previous node is pending) and one triangle test.
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
// a shared [bvh.stackDepth][kTraceBlock] array.  Returns true when the ray is
// finished (s.best: primitive id or kMissPrim; s.bt, s.b1, s.b2).
template <bool ANY, bool STATS>
__device__ __forceinline__ bool travStep(const BvhView& bvh, Trav& s, uint2* stack, TraceCounters* cnt, uint32_t* err,
                                         const uint8_t* keyLut)
{
    if (s.tg.y == 0u && s.ng.y > 0x00ffffffu)
    {
        uint32_t key = __ffs(s.ng.y >> 24) - 1;
        s.ng.y &= ~(1u << (24 + key));
        uint32_t slot  = key ^ s.oct;
        uint32_t imask = s.ng.y & 0xffu;
        uint32_t child = s.ng.x + __popc(imask & ((1u << slot) - 1u));
        if (s.ng.y > 0x00ffffffu)
        {
            if (s.sp >= int(bvh.stackDepth))
            {
                atomicOr(err, 1u);
                s.best = kMissPrim;
                return true;
            }
            stack[s.sp * kTraceBlock] = s.ng;
            ++s.sp;
        }
        uint32_t cb, tb, im;
        uint32_t hits = intersectNode(bvh.nodes, child, s.pre.o, s.inv, s.oct, s.tmin, s.bt, &cb, &tb, &im, keyLut);
        if (STATS) cnt->nodes++;
        s.ng = make_uint2(cb, (hits & 0xff000000u) | im);
        s.tg = make_uint2(tb, hits & 0x00ffffffu);
    }
    for (int tk = 0; tk < kTrisPerStep && s.tg.y; ++tk)
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
    if (s.tg.y == 0u && s.ng.y <= 0x00ffffffu)
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
                                             uint32_t* err, const uint8_t* keyLut)
{
    Trav s;
    travInit(s, o, d, tmin, tmax);
    while (!travStep<ANY, STATS>(bvh, s, stack, cnt, err, keyLut))
    {
    }
    *tHit  = s.bt;
    *b1Hit = s.b1;
    *b2Hit = s.b2;
    return s.best;
}

// ---------------------------------------------------------------------------
// Two-level traversal (CL_TWO_LEVEL).  The same node and triangle steps as
// travStep, over the top tree and, inside an instance, over its mesh's tree.
// Entering an instance pushes what is left of the top tree's current node
// (its remaining instance entries as a leaf group, y <= 0xffffff; its pending
// children as a node group, y > 0xffffff) and remembers the stack depth;
// when the mesh tree's work is done at that depth the world ray is restored
// and the top tree continues.  Hits report (instance, local triangle id).
// ---------------------------------------------------------------------------
struct Trav2
{
    RayPre        pre;
    f3            inv;
    uint32_t      oct;
    float         tmin, tmax;
    uint2         ng, tg;
    int           sp, blasSp;
    uint32_t      inst;     // current instance, kMissPrim in the top tree
    uint32_t      best, bestInst;
    float         bt, b1, b2;
    f3            wo, wd;   // the world-space ray
    const uint4*  nodes;    // the tree being traversed
    const float4* tris;
};

__device__ __forceinline__ void trav2SetRay(Trav2& s, f3 o, f3 d)
{
    s.pre   = rayPrepare(o, d);
    s.inv.x = 1.0f / (fabsf(d.x) < 1e-30f ? copysignf(1e-30f, d.x) : d.x);
    s.inv.y = 1.0f / (fabsf(d.y) < 1e-30f ? copysignf(1e-30f, d.y) : d.y);
    s.inv.z = 1.0f / (fabsf(d.z) < 1e-30f ? copysignf(1e-30f, d.z) : d.z);
    s.oct   = (s.inv.x < 0.0f ? 1u : 0u) | (s.inv.y < 0.0f ? 2u : 0u) | (s.inv.z < 0.0f ? 4u : 0u);
}

__device__ __forceinline__ void trav2Init(const BvhView& bvh, Trav2& s, f3 o, f3 d, float tmin, float tmax)
{
    trav2SetRay(s, o, d);
    s.wo = o;
    s.wd = d;
    s.tmin = tmin;
    s.tmax = tmax;
    s.ng   = make_uint2(0u, (1u << (24 + s.oct)) | 1u);
    s.tg   = make_uint2(0u, 0u);
    s.sp = s.blasSp = 0;
    s.inst  = kMissPrim;
    s.best  = s.bestInst = kMissPrim;
    s.bt    = tmax;
    s.b1 = s.b2 = 0.0f;
    s.nodes = bvh.nodes;
    s.tris  = bvh.tris;
}

// Affine map of a point (w = 1) or a direction (w = 0) by three rows.
__device__ __forceinline__ f3 xformPoint(const float4* __restrict__ m, f3 p)
{
    float4 a = __ldg(m), b = __ldg(m + 1), c = __ldg(m + 2);
    return {a.x * p.x + a.y * p.y + a.z * p.z + a.w, b.x * p.x + b.y * p.y + b.z * p.z + b.w,
            c.x * p.x + c.y * p.y + c.z * p.z + c.w};
}
__device__ __forceinline__ f3 xformDir(const float4* __restrict__ m, f3 d)
{
    float4 a = __ldg(m), b = __ldg(m + 1), c = __ldg(m + 2);
    return {a.x * d.x + a.y * d.y + a.z * d.z, b.x * d.x + b.y * d.y + b.z * d.z, c.x * d.x + c.y * d.y + c.z * d.z};
}

template <bool ANY, bool STATS>
__device__ __forceinline__ bool trav2Step(const BvhView& bvh, Trav2& s, uint2* stack, TraceCounters* cnt, uint32_t* err,
                                          const uint8_t* keyLut)
{
    if (s.tg.y == 0u && s.ng.y > 0x00ffffffu)
    {
        uint32_t key = __ffs(s.ng.y >> 24) - 1;
        s.ng.y &= ~(1u << (24 + key));
        uint32_t slot  = key ^ s.oct;
        uint32_t imask = s.ng.y & 0xffu;
        uint32_t child = s.ng.x + __popc(imask & ((1u << slot) - 1u));
        if (s.ng.y > 0x00ffffffu)
        {
            if (s.sp >= int(bvh.stackDepth))
            {
                atomicOr(err, 1u);
                s.best = kMissPrim;
                return true;
            }
            stack[s.sp * kTraceBlock] = s.ng;
            ++s.sp;
        }
        uint32_t cb, tb, im;
        uint32_t hits = intersectNode(s.nodes, child, s.pre.o, s.inv, s.oct, s.tmin, s.bt, &cb, &tb, &im, keyLut);
        if (STATS) cnt->nodes++;
        s.ng = make_uint2(cb, (hits & 0xff000000u) | im);
        s.tg = make_uint2(tb, hits & 0x00ffffffu);
    }
    if (s.tg.y)
    {
        uint32_t k = __ffs(s.tg.y) - 1;
        s.tg.y &= ~(1u << k);
        const float4* tp = s.tris + size_t(s.tg.x + k) * 3;
        if (s.inst != kMissPrim)
        {
            float4 a = __ldg(tp + 0);
            float4 b = __ldg(tp + 1);
            float4 c = __ldg(tp + 2);
            if (STATS) cnt->tris++;
            float t, u, v;
            if (intersectTri(s.pre, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, f3{c.x, c.y, c.z}, &t, &u, &v) && t > s.tmin)
            {
                uint32_t id = __float_as_uint(a.w);
                if (ANY)
                {
                    if (t < s.tmax)
                    {
                        s.bt       = t;
                        s.best     = id;
                        s.bestInst = s.inst;
                        return true;
                    }
                }
                else if (t < s.bt || (t == s.bt && (s.inst < s.bestInst || (s.inst == s.bestInst && id < s.best))))
                {
                    s.bt       = t;
                    s.best     = id;
                    s.bestInst = s.inst;
                    s.b1       = u;
                    s.b2       = v;
                }
            }
        }
        else
        {
            // An instance entry of the top tree: keep the rest of this node on the stack, enter the mesh tree.
            const uint32_t id = __float_as_uint(__ldg(&tp->w));
            const int      need = (s.ng.y > 0x00ffffffu ? 1 : 0) + (s.tg.y ? 1 : 0);
            if (s.sp + need > int(bvh.stackDepth))
            {
                atomicOr(err, 1u);
                s.best = kMissPrim;
                return true;
            }
            if (s.ng.y > 0x00ffffffu) stack[(s.sp++) * kTraceBlock] = s.ng;
            if (s.tg.y) stack[(s.sp++) * kTraceBlock] = s.tg;
            const InstDev* in = bvh.inst + id;
            s.blasSp          = s.sp;
            s.inst            = id;
            s.nodes           = in->nodes;
            s.tris            = in->tris;
            trav2SetRay(s, xformPoint(in->w2o, s.wo), xformDir(in->w2o, s.wd));
            s.ng = make_uint2(0u, (1u << (24 + s.oct)) | 1u);
            s.tg = make_uint2(0u, 0u);
            return false;
        }
    }
    if (s.tg.y == 0u && s.ng.y <= 0x00ffffffu)
    {
        if (s.inst != kMissPrim && s.sp == s.blasSp)
        {
            // The mesh tree is done: back to the top tree in world space.
            s.inst  = kMissPrim;
            s.nodes = bvh.nodes;
            s.tris  = bvh.tris;
            trav2SetRay(s, s.wo, s.wd);
        }
        if (s.sp == 0) return true;
        --s.sp;
        const uint2 e = stack[s.sp * kTraceBlock];
        if (e.y > 0x00ffffffu)
        {
            s.ng = e;
            s.tg = make_uint2(0u, 0u);
        }
        else
        {
            s.tg = e;
            s.ng = make_uint2(0u, 0u);
        }
    }
    return false;
}

// Whole two-level traversal of one ray: *inst = the hit's instance, the
// return value its triangle id within the instance's mesh (kMissPrim: none).
template <bool ANY, bool STATS>
__device__ __forceinline__ uint32_t traverse2(const BvhView& bvh, f3 o, f3 d, float tmin, float tmax, float* tHit,
                                              float* b1Hit, float* b2Hit, uint32_t* inst, uint2* stack,
                                              TraceCounters* cnt, uint32_t* err, const uint8_t* keyLut)
{
    Trav2 s;
    trav2Init(bvh, s, o, d, tmin, tmax);
    while (!trav2Step<ANY, STATS>(bvh, s, stack, cnt, err, keyLut))
    {
    }
    *tHit  = s.bt;
    *b1Hit = s.b1;
    *b2Hit = s.b2;
    *inst  = s.bestInst;
    return s.best;
}

} // namespace clb
