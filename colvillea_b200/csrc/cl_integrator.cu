// Wavefront path tracing and direct lighting on B200.
//
// Reference loop (src/core/integrators/path.cpp:84-231): per iteration, raygen
// over all pixels, then per bounce: reset queues, trace, escaped rays, shade,
// trace shadow rays, with a full host synchronisation after every launch
// (30 launches per spp).  Here the same stages run as persistent kernels over
// device-resident queues, with no host round trip per launch:
//
//   wave(cur):  kTraceClosest(rq[cur])  -> hit[]
//               kShade(rq[cur], hit[])  -> shadow queue, rq[cur^1]; finished
//                                          paths are written to the film and
//                                          their slot restarts the next camera
//                                          path (path regeneration)
//               kTraceShadow(shadows)   -> visibility per shadow ray
//               kShadowResolve          -> radiance; finishes paths whose last
//                                          vertex had a shadow ray
//               kAdvance                -> queue counters for the next wave
//
// A path's state lives in a slot (psInfo/psT/psE/psL); the ray queues hold
// slot indices and are compacted with warp-aggregated atomics (one atomicAdd
// per warp, __ballot_sync/__popc ranks), replacing the reference's one
// atomicAdd per item (libkernel/base/soa.h:39-63).  Waves are replayed from a
// CUDA graph until no path is left in flight.
//
// The per-sample arithmetic follows the reference kernels
// (src/kernel/integrators/raygeneration.cu:59-456, src/core/devices/optix.cu:112-284);
// Russian roulette is added (absent from the reference, path.cpp:135).
#include "cl_integrator.h"

#include <atomic>
#include <thread>
#include "cl_mlp_tc.cuh"

#include <chrono>
#include <cstdio>

namespace clb
{
namespace
{
constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }

// Warp-aggregated append: every lane of the warp calls it; lanes with pred
// receive consecutive indices from one atomicAdd.
__device__ __forceinline__ uint32_t warpAppend(uint32_t* counter, bool pred)
{
    uint32_t mask = __ballot_sync(kFull, pred);
    if (mask == 0u) return 0u;
    uint32_t leader = __ffs(mask) - 1u;
    uint32_t base   = 0u;
    if (laneId() == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
    base = __shfl_sync(kFull, base, leader);
    return base + __popc(mask & ((1u << laneId()) - 1u));
}

__device__ __forceinline__ uint32_t warpFetch(uint32_t* counter)
{
    uint32_t base = 0u;
    if (laneId() == 0u) base = atomicAdd(counter, 32u);
    return __shfl_sync(kFull, base, 0);
}

__device__ __forceinline__ uint32_t loadCount(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Texture slots of a material: 1-based texture indices, 0 = none.
struct MatTex
{
    uint32_t refl, rough, normal;
};

__device__ __forceinline__ Bsdf loadMaterial(const float4* mats, uint32_t m, MatTex* tx)
{
    float4 a = __ldg(mats + kMatF4 * m), b = __ldg(mats + kMatF4 * m + 1), c = __ldg(mats + kMatF4 * m + 2);
    uint4  d = __ldg(reinterpret_cast<const uint4*>(mats + kMatF4 * m + 3));
    tx->refl   = d.x;
    tx->rough  = d.y;
    tx->normal = d.z;
    Bsdf   s;
    s.type   = __float_as_uint(a.x);
    s.r      = {a.y, a.z, a.w};
    s.alpha  = b.x;
    s.etaInt = b.y;
    s.eta    = {b.z, b.w, c.x};
    s.k      = {c.y, c.z, c.w};
    return s;
}

__device__ __forceinline__ float4 texLookup(const unsigned long long* tex, uint32_t oneBased, f2 uv)
{
    return tex2D<float4>(cudaTextureObject_t(__ldg(tex + (oneBased - 1u))), uv.x, uv.y);
}

// Material::getBSDF(uv) (material.h:93-108): a reflectance texture replaces
// the constant reflectance (diffusemtl.h:22-27, metal.h:40-45); a roughness
// texture's red channel replaces the roughness, squared to alpha (metal.h:47-52).
__device__ __forceinline__ void applyTextures(const unsigned long long* tex, const MatTex& tx, f2 uv, Bsdf* b)
{
    if (tx.refl)
    {
        float4 c = texLookup(tex, tx.refl, uv);
        b->r     = {c.x, c.y, c.z};
    }
    if (tx.rough)
    {
        float r  = texLookup(tex, tx.rough, uv).x;
        b->alpha = r * r;
    }
}

struct HitAttr
{
    f3       p, ng, ns, dpdu, dpdv;
    f2       uv;
    uint32_t material;
};

// Closest-hit attributes (optix.cu:137-227) of a triangle given by its
// vertex ids and material (ti, the triangle's triIdx entry).
// Two-level scenes: ti.w is the instance; the vertices are the mesh's, in
// object space, and the attributes are mapped to world space before the
// shading frame is built (position by the instance transform, normals by the
// inverse transpose - the rows of object-from-world read as columns -, the
// geometric normal flipped for a mirroring transform, tangents by the linear
// part).  The flattened path (sc.inst null) keeps world-space vertices.
__device__ __forceinline__ f3 xformNormal(const float4* __restrict__ w2o, f3 n)
{
    float4 a = __ldg(w2o), b = __ldg(w2o + 1), c = __ldg(w2o + 2);
    return {a.x * n.x + b.x * n.y + c.x * n.z, a.y * n.x + b.y * n.y + c.y * n.z, a.z * n.x + b.z * n.y + c.z * n.z};
}

__device__ __forceinline__ HitAttr hitAttributesTri(const SceneDev& sc, uint4 ti, float b1, float b2)
{
    const InstDev* ip = sc.bvh.inst ? sc.bvh.inst + ti.w : nullptr;
    float4  a0 = __ldg(sc.vtx + 3 * size_t(ti.x)), a1 = __ldg(sc.vtx + 3 * size_t(ti.x) + 1), a2 = __ldg(sc.vtx + 3 * size_t(ti.x) + 2);
    float4  c0 = __ldg(sc.vtx + 3 * size_t(ti.y)), c1 = __ldg(sc.vtx + 3 * size_t(ti.y) + 1), c2 = __ldg(sc.vtx + 3 * size_t(ti.y) + 2);
    float4  e0 = __ldg(sc.vtx + 3 * size_t(ti.z)), e1 = __ldg(sc.vtx + 3 * size_t(ti.z) + 1), e2 = __ldg(sc.vtx + 3 * size_t(ti.z) + 2);
    f3      p0{a0.x, a0.y, a0.z}, p1{c0.x, c0.y, c0.z}, p2{e0.x, e0.y, e0.z};
    uint32_t flags = __float_as_uint(a2.w);
    float   b0    = 1.0f - b1 - b2;
    HitAttr h;
    h.material = ip ? __ldg(&ip->material) : ti.w;
    h.p        = b0 * p0 + b1 * p1;
    h.p        = h.p + b2 * p2;
    if (flags & 2u)
        h.uv = {b0 * a2.y + b1 * c2.y + b2 * e2.y, b0 * a2.z + b1 * c2.z + b2 * e2.z};
    else
        h.uv = {b0, b1};
    f3 Ng = cross(p1 - p0, p2 - p0);
    if (ip)
    {
        h.p = xformPoint(ip->o2w, h.p);
        Ng  = xformNormal(ip->w2o, Ng);
        if (__ldg(&ip->flags) & 1u) Ng = -Ng;
    }
    Ng = normalize(Ng);
    f3 Ns;
    if (flags & 1u)
    {
        f3 n = b0 * f3{a0.w, a1.x, a1.y} + b1 * f3{c0.w, c1.x, c1.y};
        n    = n + b2 * f3{e0.w, e1.x, e1.y};
        if (ip) n = xformNormal(ip->w2o, n);
        Ns = normalize(n);
    }
    else
        Ns = normalize(Ng);
    if (dot(Ns, Ns) == 0.0f) Ns = Ng;
    if (dot(Ng, Ns) < 0.0f) Ng = -Ng;
    f3 t    = b0 * f3{a1.z, a1.w, a2.x} + b1 * f3{c1.z, c1.w, c2.x};
    t       = t + b2 * f3{e1.z, e1.w, e2.x};
    if (ip) t = xformDir(ip->o2w, t);
    f3 dpdu = normalize(t);
    f3 dpdv{0.0f, 0.0f, 0.0f};
    if (dot(dpdu, dpdu) > 0.0f)
    {
        dpdv = cross(Ns, dpdu);
        if (dot(dpdv, dpdv) > 0.0f)
        {
            dpdv = normalize(dpdv);
            dpdu = cross(dpdv, Ns);
        }
        else
            makeFrame(Ns, &dpdu, &dpdv);
    }
    else
        makeFrame(Ns, &dpdu, &dpdv);
    h.ng   = Ng;
    h.ns   = Ns;
    h.dpdu = dpdu;
    h.dpdv = dpdv;
    return h;
}

// Camera path start (generateCameraRays, raygeneration.cu:83-102): path index
// p -> pixel p mod W*H, frame frame0 + p / (W*H).
__device__ __forceinline__ void startPath(const Params& P, const WaveParams& wp, uint32_t slot, unsigned long long p,
                                          int q, uint32_t idx)
{
    unsigned long long wh = (unsigned long long)wp.W * wp.H;
    uint32_t pix   = uint32_t(p % wh);
    uint32_t frame = wp.frame0 + uint32_t(p / wh);
    uint32_t px = pix % wp.W, py = pix / wp.W;
    Rng      rng{px, py, frame, 0u};
    f2       j = rng.next2D();
    f2       screen{(float(px) + j.x) / float(wp.W), (float(py) + j.y) / float(wp.H)};
    f3       pos{wp.cam[0], wp.cam[1], wp.cam[2]}, d00{wp.cam[3], wp.cam[4], wp.cam[5]};
    f3       ddu{wp.cam[6], wp.cam[7], wp.cam[8]}, ddv{wp.cam[9], wp.cam[10], wp.cam[11]};
    f3       d = d00 + screen.x * ddu;
    d          = d + screen.y * ddv;
    d          = normalize(d);
    P.q.psInfo[slot]   = make_uint4(pix, frame, 1u | (rng.ctr << 8), 0u);
    P.q.psT[slot]      = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    // Radiance cache: one path in trainMask + 1 (Fibonacci hash of the path
    // index) is a training path.
    const bool train = wp.cacheTrain && ((uint32_t((p * 0x9E3779B97F4A7C15ull) >> 40) & P.c.trainMask) == 0u);
    P.q.psE[slot]      = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(train ? kCacheTrainBit : 0u));
    P.q.psL[slot]      = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.q.rqO[q][idx]    = make_float4(pos.x, pos.y, pos.z, 0.0f);
    P.q.rqD[q][idx]    = make_float4(d.x, d.y, d.z, FLT_MAX);
    P.q.rqSlot[q][idx] = slot;
}

// Guided path tracing: training records of a finished path.  Recorded vertex
// k holds the throughput T_k that reached it and the path radiance L_k after
// its own emitter sample; (L - L_k) / T_k estimates f |cos| L_i / p of the
// direction sampled at k, whose luminance is the record's weight.
__device__ __noinline__ void flushRecords(GuideDev g, const uint4* psInfo, Counters* ctr, uint32_t slot,
                                          uint32_t stride, float lx, float ly, float lz)
{
    uint32_t mask = psInfo[slot].w;
    const float4* h = g.hist + size_t(slot / stride) * g.histDepth * kHistF4;
    while (mask)
    {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1u;
        const float4* e  = h + k * kHistF4;
        float4        e0 = e[0], e1 = e[1], e2 = e[2], e3 = e[3], e4 = e[4];
        float         w  = 0.0f;
        if (e0.w > 0.0f) w += 0.2126f * (lx - e4.x) / e0.w;
        if (e1.w > 0.0f) w += 0.7152f * (ly - e4.y) / e1.w;
        if (e2.w > 0.0f) w += 0.0722f * (lz - e4.z) / e2.w;
        if (!(w > 0.0f) || !(w < FLT_MAX)) continue;
        uint32_t idx = atomicAdd(&ctr->recCount, 1u);
        if (idx >= g.recCap) continue;
        float4* r = g.rec + size_t(idx) * kRecordF4;
        r[0]      = make_float4(e0.x, e0.y, e0.z, w);
        r[1]      = make_float4(e1.x, e1.y, e1.z, 0.0f);
        r[2]      = make_float4(e2.x, e2.y, e2.z, 0.0f);
        r[3]      = make_float4(e3.x, e3.y, e3.z, e3.w);
    }
}

// Radiance cache: training records of a finished training path.  Recorded
// vertex k holds the throughput T_k that reached it and the path radiance
// L_k before its emitter sample; (L - L_k) / T_k is the radiance the path
// gathered from k on, an estimate of the outgoing radiance at k.
__device__ __noinline__ void flushCacheRecords(CacheDev c, const float4* psE, Counters* ctr, uint32_t slot, float lx,
                                               float ly, float lz)
{
    uint32_t      mask = __float_as_uint(psE[slot].w) & ~kCacheTrainBit;
    const float4* h    = c.hist + size_t(slot) * c.histDepth * kCacheHistF4;
    while (mask)
    {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1u;
        const float4* e  = h + k * kCacheHistF4;
        float4        e0 = e[0], e1 = e[1], e2 = e[2], e3 = e[3];
        if (!(e0.w > 0.0f) || !(e1.w > 0.0f) || !(e2.w > 0.0f)) continue;
        float ty = fmaxf((lx - e3.x) / e0.w, 0.0f), tg = fmaxf((ly - e3.y) / e1.w, 0.0f),
              tb = fmaxf((lz - e3.z) / e2.w, 0.0f);
        if (!(ty < FLT_MAX) || !(tg < FLT_MAX) || !(tb < FLT_MAX)) continue;
        uint32_t idx = atomicAdd(&ctr->cacheRec, 1u);
        if (idx >= c.recCap) continue;
        float4* r = c.rec + size_t(idx) * kRecordF4;
        r[0]      = make_float4(e0.x, e0.y, e0.z, 1.0f);
        r[1]      = make_float4(e1.x, e1.y, e1.z, 0.0f);
        r[2]      = make_float4(e2.x, e2.y, e2.z, 0.0f);
        r[3]      = make_float4(ty, tg, tb, 0.0f);
    }
}

// Film write of finished paths, then regeneration of their slots.  Called by
// every lane of the warp.
__device__ __forceinline__ void finishPaths(const Params& P, const WaveParams& wp, int nxt, bool finish, uint32_t slot,
                                            f3 L)
{
    if (finish && wp.recStride && slot % wp.recStride == 0u)
        flushRecords(P.g, P.q.psInfo, P.q.ctr, slot, wp.recStride, L.x, L.y, L.z);
    if (finish && wp.cacheTrain && (__float_as_uint(P.q.psE[slot].w) & ~kCacheTrainBit))
        flushCacheRecords(P.c, P.q.psE, P.q.ctr, slot, L.x, L.y, L.z);
    if (finish)
    {
        uint32_t pix = P.q.psInfo[slot].x;
        float*   f   = reinterpret_cast<float*>(P.q.film + pix);
        atomicAdd(f + 0, L.x);
        atomicAdd(f + 1, L.y);
        atomicAdd(f + 2, L.z);
        if (P.q.film64)
        {
            double* g = P.q.film64 + 6 * size_t(pix);
            atomicAdd(g + 0, double(L.x));
            atomicAdd(g + 1, double(L.y));
            atomicAdd(g + 2, double(L.z));
            atomicAdd(g + 3, double(L.x) * double(L.x));
            atomicAdd(g + 4, double(L.y) * double(L.y));
            atomicAdd(g + 5, double(L.z) * double(L.z));
        }
    }
    uint32_t mask = __ballot_sync(kFull, finish);
    if (mask == 0u) return;
    uint32_t           leader = __ffs(mask) - 1u;
    unsigned long long base   = 0ull;
    if (laneId() == leader) base = atomicAdd(&P.q.ctr->pathNext, (unsigned long long)__popc(mask));
    base                  = __shfl_sync(kFull, base, leader);
    unsigned long long p  = base + __popc(mask & ((1u << laneId()) - 1u));
    bool               gen = finish && p < wp.totalPaths;
    uint32_t           idx = warpAppend(&P.q.ctr->rayCount[nxt], gen);
    if (gen)
    {
        if (idx < P.q.slots)
            startPath(P, wp, slot, p, nxt, idx);
        else
            atomicOr(&P.q.ctr->error, 8u);
    }
}

__device__ __forceinline__ f3 ld3(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float maxComp(f3 v)
{
    float m = v.x;
    if (v.y > m) m = v.y;
    if (v.z > m) m = v.z;
    return m;
}

} // namespace

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ void warpStats(const TraceCounters& tc, unsigned long long* nodes, unsigned long long* tris)
{
    unsigned long long a = tc.nodes, b = tc.tris;
    for (int o = 16; o > 0; o >>= 1)
    {
        a += __shfl_xor_sync(kFull, a, o);
        b += __shfl_xor_sync(kFull, b, o);
    }
    if (laneId() == 0)
    {
        atomicAdd(nodes, a);
        atomicAdd(tris, b);
    }
}

// Resident blocks per SM of the traversal kernels.  Flattened scenes: 7
// (72 registers; 8 blocks at 64 registers was 3% slower on config 2 with the
// lane refill, 6 blocks the same as 7).  Two-level scenes: 5 (their state is
// larger; 8 blocks would spill).
constexpr int kTraceBlocksFlat = 7;
constexpr int kTraceBlocksTwo  = 5;

struct ClassifyView
{
    const uint4* __restrict__ triIdx;
    const float4* __restrict__ mats;
    uint32_t* classIdx;
    uint32_t  cap;
    uint4*    hitIdx; // per ray: the hit triangle's triIdx entry (vertex ids, material), for the shading kernels
    uint32_t* hitInst; // two-level scenes: per ray, the hit's instance (kTraceClosest -> kClassifyHits)
};

constexpr int kClassEscaped = 3;

// Shading class of a finished closest-hit ray (-1: none), with the hit's
// triangle index entry written for the shading kernels.
template <bool TWO>
__device__ __forceinline__ int classifyHit(const BvhView& bvh, const ClassifyView& cv, uint32_t i, uint32_t prim,
                                           uint32_t inst, uint32_t loc)
{
    if (prim == kMissPrim) return kClassEscaped;
    if (TWO)
    {
        const InstDev* ip = bvh.inst + inst;
        uint4          ti = __ldg(&cv.triIdx[__ldg(&ip->triBase) + loc]);
        ti.w              = inst;
        cv.hitIdx[i]      = ti;
        return int(__float_as_uint(__ldg(&cv.mats[kMatF4 * __ldg(&ip->material)].x)));
    }
    const uint4 ti = __ldg(&cv.triIdx[prim]);
    cv.hitIdx[i]   = ti;
    return int(__float_as_uint(__ldg(&cv.mats[kMatF4 * ti.w].x)));
}

// Warp-local supply of queue entries for the persistent traversal kernels.
// A warp takes 32 consecutive entries per atomicAdd and hands them to its
// idle lanes in lane order, so that a lane whose ray has finished takes the
// next ray while the others continue (the warp no longer waits for its
// longest ray), and the rays of a warp stay within a few chunks of the queue.
// The warp's unstarted entries [x, y) live in shared memory (they are only
// touched when lanes are refilled); x = kMissPrim: the queue is exhausted.
__device__ __forceinline__ void supplyInit(uint2* ws)
{
    if (laneId() == 0u) *ws = make_uint2(0u, 0u);
    __syncwarp();
}

// Every lane calls it with the same `want` (the lanes to supply); returns
// the supplied lane's entry, kMissPrim for the others.
__device__ __forceinline__ uint32_t supplyLanes(uint2* ws, uint32_t* fetch, uint32_t n, uint32_t want)
{
    const uint32_t lane = laneId(), lt = (1u << lane) - 1u;
    uint2          w    = *ws;
    uint32_t       item = kMissPrim;
    while (want && w.x != kMissPrim)
    {
        if (w.x >= w.y)
        {
            const uint32_t nb = warpFetch(fetch);
            w                 = nb >= n ? make_uint2(kMissPrim, kMissPrim) : make_uint2(nb, min(nb + 32u, n));
            if (nb >= n) break;
        }
        const uint32_t avail = w.y - w.x, r = __popc(want & lt);
        const bool     mine  = (want >> lane) & 1u;
        if (mine && r < avail) item = w.x + r;
        w.x += min(uint32_t(__popc(want)), avail);
        want = __ballot_sync(kFull, mine && r >= avail);
    }
    __syncwarp();
    if (lane == 0u) *ws = w;
    __syncwarp();
    return item;
}

// Ray indices of the wave queues stay below this (kTraceClosest and the
// shadow kernel keep kMissPrim as their idle-lane mark).
constexpr uint32_t kMaxPathSlots = 0x0fffffffu;

// Traversal state of a flattened (Trav) or two-level (Trav2) scene.
template <bool TWO> struct TravOf
{
    using T = Trav;
};
template <> struct TravOf<true>
{
    using T = Trav2;
};

// Closest-hit traversal of a ray queue by persistent warps: each lane
// traverses one ray at a time and takes the next from the warp's supply when
// it finishes.  The hits' shading classes are appended by kClassifyHits
// afterwards, in ray order (a class lookup inside the step loop would stall
// the whole warp on one lane's dependent gathers).  CLASSIFY: the launch is
// a wave's (kClassifyHits follows); without it the hits are final (the ray
// query entry points).  TWO: two-level scene (CL_TWO_LEVEL); with CLASSIFY a
// hit holds the instance-local triangle id and cv.hitInst its instance, which
// kClassifyHits turns into the global id and the triangle index entry
// (object-space vertex ids, the instance in .w).
template <bool STATS, bool CLASSIFY, bool TWO = false>
__global__ void __launch_bounds__(kTraceBlock, TWO ? kTraceBlocksTwo : kTraceBlocksFlat) kTraceClosest(BvhView bvh, const float4* __restrict__ O,
                                                                const float4* __restrict__ D, const uint32_t* count,
                                                                uint32_t* fetch, float4* __restrict__ hitOut,
                                                                Counters* ctr, ClassifyView cv)
{
    extern __shared__ uint2 stack[];
    __shared__ uint8_t      keyLut[kKeyLutBytes];
    __shared__ uint2        supply[kTraceBlock / 32];
    fillKeyLut(keyLut);
    const uint32_t   n = loadCount(count);
    TraceCounters    tc{0u, 0u};
    // Idle lanes are refilled once at least kRefillIdle of them are idle.
    uint2* ws = supply + (threadIdx.x >> 5);
    supplyInit(ws);
    typename TravOf<TWO>::T s;
    uint32_t                ray = kMissPrim;
    for (;;)
    {
        const uint32_t idle = __ballot_sync(kFull, ray == kMissPrim);
        if (uint32_t(__popc(idle)) >= kRefillIdle)
        {
            if (ws->x != kMissPrim)
            {
                const uint32_t item = supplyLanes(ws, fetch, n, idle);
                if (item != kMissPrim)
                {
                    ray            = item;
                    const float4 o = O[item], d = D[item];
                    if constexpr (TWO)
                        trav2Init(bvh, s, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, o.w, d.w);
                    else
                        travInit(s, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, o.w, d.w);
                }
            }
            if (__all_sync(kFull, ray == kMissPrim)) break;
        }
        if (ray != kMissPrim)
            for (uint32_t k = 0; k < kRefillSteps; ++k)
            {
                bool done;
                if constexpr (TWO)
                    done = trav2Step<false, STATS>(bvh, s, stack + threadIdx.x, &tc, &ctr->error, keyLut);
                else
                    done = travStep<false, STATS>(bvh, s, stack + threadIdx.x, &tc, &ctr->error, keyLut);
                if (done)
                {
                    if constexpr (TWO)
                    {
                        if (CLASSIFY)
                        {
                            // The instance-local id; kClassifyHits makes it global.
                            hitOut[ray]     = make_float4(s.bt, __uint_as_float(s.best), s.b1, s.b2);
                            cv.hitInst[ray] = s.bestInst;
                        }
                        else
                        {
                            const uint32_t prim =
                                s.best == kMissPrim ? kMissPrim : __ldg(&bvh.inst[s.bestInst].primBase) + s.best;
                            hitOut[ray] = make_float4(s.bt, __uint_as_float(prim), s.b1, s.b2);
                        }
                    }
                    else
                        hitOut[ray] = make_float4(s.bt, __uint_as_float(s.best), s.b1, s.b2);
                    ray = kMissPrim;
                    break;
                }
            }
    }
    if (STATS) warpStats(tc, &ctr->statNodes, &ctr->statTris);
}

// Shading classes of a wave's closest hits.  A block
// takes tiles of kClassifyTile consecutive rays (kClassifyPer per thread,
// in ray order), counts each class over the tile with warp ballots and a
// block scan, reserves the tile's range of each class queue with one
// atomicAdd per class, and writes the rays there in ray order; the hit's
// triangle index entry is written for the shading kernels.  Two-level
// scenes (TWO): the hit's instance-local triangle id and instance (from
// kTraceClosest) become the global id, written back into the hit.
// Grid-stride over the wave's ray count (read on the device).
constexpr int kClassifyThreads = 256;
constexpr int kClassifyPer     = 4;
constexpr int kClassifyTile    = kClassifyThreads * kClassifyPer;
template <bool TWO>
__global__ void __launch_bounds__(kClassifyThreads) kClassifyHits(BvhView bvh, float4* hit, const uint32_t* count,
                                                                  Counters* ctr, ClassifyView cv)
{
    constexpr int  kWarps = kClassifyThreads / 32;
    __shared__ uint32_t wcount[kClassifyPer][kWarps][4]; // rays of class c in (round r, warp w)
    __shared__ uint32_t cbase[4];
    const uint32_t n = loadCount(count);
    const uint32_t w = threadIdx.x >> 5, lane = laneId(), lt = (1u << lane) - 1u;
    for (uint32_t tile = blockIdx.x * uint32_t(kClassifyTile); tile < n; tile += gridDim.x * uint32_t(kClassifyTile))
    {
        int cls[kClassifyPer];
#pragma unroll
        for (int r = 0; r < kClassifyPer; ++r)
        {
            const uint32_t i = tile + uint32_t(r * kClassifyThreads) + threadIdx.x;
            cls[r]           = -1;
            if (i < n)
            {
                const uint32_t h = __float_as_uint(hit[i].y);
                if constexpr (TWO)
                {
                    const uint32_t inst = cv.hitInst[i];
                    const uint32_t prim = h == kMissPrim ? kMissPrim : __ldg(&bvh.inst[inst].primBase) + h;
                    hit[i].y            = __uint_as_float(prim);
                    cls[r]              = classifyHit<true>(bvh, cv, i, prim, inst, h);
                }
                else
                    cls[r] = classifyHit<false>(bvh, cv, i, h, 0u, 0u);
            }
        }
        uint32_t rank[kClassifyPer];
#pragma unroll
        for (int r = 0; r < kClassifyPer; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                const uint32_t m = __ballot_sync(kFull, cls[r] == c);
                if (cls[r] == c) rank[r] = __popc(m & lt);
                if (lane == 0u) wcount[r][w][c] = __popc(m);
            }
        __syncthreads();
        // Exclusive scan over (round, warp) per class, in ray order, by the first 4 threads; then the reservation.
        if (threadIdx.x < 4u)
        {
            const int c   = int(threadIdx.x);
            uint32_t  sum = 0u;
            for (int r = 0; r < kClassifyPer; ++r)
                for (int k = 0; k < kWarps; ++k)
                {
                    const uint32_t v = wcount[r][k][c];
                    wcount[r][k][c]  = sum;
                    sum += v;
                }
            cbase[c] = sum ? atomicAdd(&ctr->classCount[c], sum) : 0u;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kClassifyPer; ++r)
            if (cls[r] >= 0)
            {
                const uint32_t i = tile + uint32_t(r * kClassifyThreads) + threadIdx.x;
                const uint32_t k = cbase[cls[r]] + wcount[r][w][cls[r]] + rank[r];
                if (k < cv.cap)
                    cv.classIdx[size_t(cls[r]) * cv.cap + k] = i;
                else
                    atomicOr(&ctr->error, 8u);
            }
        __syncthreads();
    }
}

// Shadow rays (any hit) of the shadow queue.  Item k is entry k (path
// tracing) or ray k&1 of entry k>>1 (direct lighting, two rays per entry).
// vis[k] = 1 when the ray reaches its light, 0 otherwise.
template <bool DL, bool STATS, bool TWO = false>
__global__ void __launch_bounds__(kTraceBlock, TWO ? kTraceBlocksTwo : kTraceBlocksFlat) kTraceShadow(Params P)
{
    extern __shared__ uint2 stack[];
    __shared__ uint8_t      keyLut[kKeyLutBytes];
    __shared__ uint2        supply[kTraceBlock / 32];
    fillKeyLut(keyLut);
    const uint32_t   n = loadCount(&P.q.ctr->shadowCount) * (DL ? 2u : 1u);
    TraceCounters    tc{0u, 0u};
    // Idle lanes refilled as in kTraceClosest.
    uint2* ws = supply + (threadIdx.x >> 5);
    supplyInit(ws);
    typename TravOf<TWO>::T s;
    uint32_t                ray = kMissPrim;
    for (;;)
    {
        const uint32_t idle = __ballot_sync(kFull, ray == kMissPrim);
        if (uint32_t(__popc(idle)) >= kRefillIdle)
        {
            if (ws->x != kMissPrim)
            {
                const uint32_t item = supplyLanes(ws, &P.q.ctr->fetchShadow, n, idle);
                if (item != kMissPrim)
                {
                    const uint32_t e  = DL ? item >> 1 : item;
                    const float4   o4 = P.q.sqO[e];
                    const float4   d4 = (DL && (item & 1u)) ? P.q.sqD2[e] : P.q.sqD[e];
                    if (d4.w != 0.0f)
                    {
                        ray = item;
                        if constexpr (TWO)
                            trav2Init(P.sc.bvh, s, f3{o4.x, o4.y, o4.z}, f3{d4.x, d4.y, d4.z}, kRayEps, FLT_MAX);
                        else
                            travInit(s, f3{o4.x, o4.y, o4.z}, f3{d4.x, d4.y, d4.z}, kRayEps, FLT_MAX);
                    }
                    else
                        P.q.vis[item] = 0; // no emitter sample on this entry
                }
            }
            if (__all_sync(kFull, ray == kMissPrim) && ws->x == kMissPrim) break;
        }
        if (ray != kMissPrim)
            for (uint32_t k = 0; k < kRefillSteps; ++k)
            {
                bool done;
                if constexpr (TWO)
                    done = trav2Step<true, STATS>(P.sc.bvh, s, stack + threadIdx.x, &tc, &P.q.ctr->error, keyLut);
                else
                    done = travStep<true, STATS>(P.sc.bvh, s, stack + threadIdx.x, &tc, &P.q.ctr->error, keyLut);
                if (done)
                {
                    P.q.vis[ray] = s.best == kMissPrim ? 1 : 0;
                    ray          = kMissPrim;
                    break;
                }
            }
    }
    if (STATS) warpStats(tc, &P.q.ctr->statNodesS, &P.q.ctr->statTrisS);
}

// CMP: 1 = the reference's estimator (all CL_COMPAT_* flags), 0 = the
// corrected one, 2 = a mix read at run time; ALIAS: alias-table dome sampling.
// MAT: the shading class this launch serves (BSDF type 0-2, or 3 = escaped
// rays), from the class queues written by kTraceClosest; -1 = every ray of
// the ray queue.  Specialising keeps each instantiation free of the other
// modes' and materials' code.
// GUIDE (path tracing, corrected estimator, BSDF classes): one-sample MIS of
// the BSDF and the network's vMF mixture for this ray (kGuideMlp), which is
// sampled with probability a = the sum of its lobe weights (1 - bsdf_fraction,
// or learned); every pdf of the BSDF strategy - emitter-sample MIS, the
// throughput update and the escaped-ray MIS - becomes (1 - a) p_bsdf + a p_guide.
template <bool DL, int CMP, bool ALIAS, int MAT, bool GUIDE = false>
__global__ void __launch_bounds__(128) kShade(Params P, int cur)
{
    const WaveParams wp = *P.wp;
    const SceneDev&  sc = P.sc;
    const uint32_t   n  = MAT < 0 ? loadCount(&P.q.ctr->rayCount[cur]) : loadCount(&P.q.ctr->classCount[MAT < 0 ? 0 : MAT]);
    const int        nxt = cur ^ 1;
    // The guided mixture pdf needs the sampling densities of the BSDF: a
    // guided kernel never takes the reference's pdf functions (setGuiding also
    // refuses every CL_COMPAT_* flag).
    const bool compatPdf   = !GUIDE && (CMP == 2 ? (wp.flags & CL_COMPAT_PDF) != 0 : CMP == 1);
    const bool compatFrame = CMP == 2 ? (wp.flags & CL_COMPAT_FRAME) != 0 : CMP == 1;
    const bool compatEsc   = CMP == 2 ? (wp.flags & CL_COMPAT_ESCAPE) != 0 : CMP == 1;
    const bool alias       = ALIAS;
    const uint32_t N       = sc.numEmitters;
    // Static assignment of 32-ray batches to warps (grid-stride): a dynamic
    // fetch would put a same-address atomicAdd at the head of every batch's
    // chain of dependent gathers.
    const uint32_t gw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32u; base < n; base += gw * 32u)
    {
        uint32_t i     = base + laneId();
        bool     valid = i < n;
        if (MAT >= 0 && valid) i = P.q.classIdx[size_t(MAT) * P.q.slots + i];
        bool     pushShadow = false, shadow1 = false, shadow2 = false, pushRay = false, finish = false;
        uint32_t slot = 0u, info2 = 0u, recBit = 0u, vDepth = 0u, cst = 0u;
        f3       tIn{0, 0, 0};
        f3       L{0, 0, 0}, T{1, 1, 1}, E{0, 0, 0}, pHit{0, 0, 0}, sdir{0, 0, 0}, Li{0, 0, 0}, sdir2{0, 0, 0},
            Ld{0, 0, 0}, ndir{0, 0, 0};
        if (valid)
        {
            slot          = P.q.rqSlot[cur][i];
            float4 hh     = P.q.hit[i];
            uint4  ti     = MAT == kClassEscaped ? make_uint4(0u, 0u, 0u, 0u) : P.q.hitIdx[i];
            float4 rd     = P.q.rqD[cur][i];
            // Surface classes: the hit exists, so its vertex gathers start with the
            // path-state loads instead of after the depth tests that need them.
            HitAttr a0{};
            if constexpr (MAT >= 0 && MAT != kClassEscaped) a0 = hitAttributesTri(sc, ti, hh.z, hh.w);
            uint4  info   = P.q.psInfo[slot];
            uint32_t depth = info.z & 0xffu;
            vDepth         = depth;
            Rng    rng{info.x % wp.W, info.x / wp.W, info.y, info.z >> 8};
            T             = ld3(P.q.psT[slot]);
            float4 e4     = P.q.psE[slot];
            E             = ld3(e4);
            cst           = __float_as_uint(e4.w);
            L             = ld3(P.q.psL[slot]);
            f3       d    = ld3(rd);
            uint32_t prim = __float_as_uint(hh.y);
            if (MAT == kClassEscaped || (MAT < 0 && prim == kMissPrim))
            {
                // evaluateEscapedRays (raygeneration.cu:105-136)
                if (sc.hasDome)
                {
                    f3 Le = domeEval(sc.dome, d, !compatEsc);
                    if (depth == 1u)
                        L = L + Le;
                    else if (compatEsc)
                        L = L + T * (Le * E);
                    else
                    {
                        float pd = domePdf(sc.dome, d, true) / float(N);
                        float w  = E.x / (E.x + pd);
                        L        = L + T * (Le * w);
                    }
                }
                finish = true;
            }
            else if (!DL && P.c.termDepth && depth == P.c.termDepth && !(cst & kCacheTrainBit))
            {
                // The path ends in the radiance cache (kCacheMlp's prediction).
                float4 cl = P.c.L[i];
                L         = L + T * f3{cl.x, cl.y, cl.z};
                finish    = true;
            }
            else if (!DL && depth == wp.maxDepth)
                finish = true;
            else
            {
                HitAttr a    = (MAT >= 0 && MAT != kClassEscaped) ? a0 : hitAttributesTri(sc, ti, hh.z, hh.w);
                MatTex  tx;
                Bsdf    bsdf = loadMaterial(sc.mats, a.material, &tx);
                if (tx.refl | tx.rough) applyTextures(sc.tex, tx, a.uv, &bsdf);
                if (!DL && (cst & kCacheTrainBit) && wp.cacheTrain && depth <= P.c.histDepth)
                {
                    // Radiance-cache training path: vertex history (flushCacheRecords).
                    float4* h = P.c.hist + (size_t(slot) * P.c.histDepth + depth - 1u) * kCacheHistF4;
                    f3 pn = (a.p - f3{P.g.boxMin[0], P.g.boxMin[1], P.g.boxMin[2]}) * P.g.boxScale;
                    h[0]  = make_float4(pn.x, pn.y, pn.z, T.x);
                    h[1]  = make_float4(a.ns.x, a.ns.y, a.ns.z, T.y);
                    h[2]  = make_float4(-d.x, -d.y, -d.z, T.z);
                    h[3]  = make_float4(L.x, L.y, L.z, 0.0f);
                    cst |= 1u << (depth - 1u);
                    reinterpret_cast<uint32_t*>(P.q.psE + slot)[3] = cst;
                }
                if (MAT >= 0) bsdf.type = uint32_t(MAT);
                pHit         = a.p;
                f3    wo     = -d;
                guide::Lobes G;
                float        gf = 1.0f; // probability of BSDF sampling: 1 - sum of the lobe weights
                // Vertices shallower than the guide's minimum depth were not inferred, and near-specular
                // ones (GGX alpha below the guide's minimum) are not guided: BSDF sampling alone (zero
                // lobe weights), no training record.
                const bool guided =
                    GUIDE && depth >= P.g.minDepth && (bsdf.type == kDiffuse || bsdf.alpha >= P.g.minAlpha);
                if (GUIDE && !guided)
#pragma unroll
                    for (int k = 0; k < guide::kLobes; ++k)
                    {
                        G.l[k] = make_float4(0.0f, 0.0f, 1.0f, 1.0f);
                        G.w[k] = 0.0f;
                    }
                if (guided)
                {
                    const float4* lb = P.g.lobes + size_t(i) * kLobeF4;
#pragma unroll
                    for (int k = 0; k < guide::kLobes; ++k) G.l[k] = lb[k];
                    float4 w0 = lb[8], w1 = lb[9];
                    G.w[0] = w0.x, G.w[1] = w0.y, G.w[2] = w0.z, G.w[3] = w0.w;
                    G.w[4] = w1.x, G.w[5] = w1.y, G.w[6] = w1.z, G.w[7] = w1.w;
                    gf = 1.0f - (((w0.x + w0.y) + (w0.z + w0.w)) + ((w1.x + w1.y) + (w1.z + w1.w)));
                }
                f2    u      = rng.next2D();
                // Shading frame (Material::getShadingFrame, material.h:128-147).
                // Path tracing passes (ng, ns) swapped (raygeneration.cu:324-330):
                // without a normal map the frame's normal is then the geometric
                // one (the compat quirk); with one, the map's tangent frame and
                // the pull-up use the shading normal, kept in both estimators.
                // The reference's direct-lighting kernel builds {dpdv, dpdu, ns}
                // itself and ignores normal maps (raygeneration.cu:179,237).
                Frame fr;
                if (tx.normal && !(DL && compatFrame))
                {
                    float4 nt = texLookup(sc.tex, tx.normal, a.uv);
                    fr = normalMappedFrame(wo, a.dpdu, a.dpdv, a.ns, f3{nt.x, nt.y, nt.z}, bsdf.type != kDielectric);
                }
                else
                    fr = Frame{a.dpdv, a.dpdu, (!DL && compatFrame) ? a.ng : a.ns};
                // Emitter sampling with MIS (raygeneration.cu:332-384 / 174-227).
                if (N > 0u)
                {
                    uint32_t pick = min(uint32_t(floorf(u.x * float(N))), N - 1u);
                    f2       us{u.x * float(N) - float(pick), u.y};
                    f3       ldir{0, 0, 0};
                    float    lpdf = 0.0f;
                    const EmitterDev& em = sc.emitters[pick];
                    f3 value = em.type == 0u ? directionalSample(em.dl, us, &ldir, &lpdf)
                                             : domeSample(sc.dome, us, alias, &ldir, &lpdf);
                    if (compatEsc) value = value * float(N);
                    if (lpdf == 0.0f) value = {0.0f, 0.0f, 0.0f};
                    if (nonzero(value) && lpdf > 0.0f)
                    {
                        f3 wiL = fr.toLocal(ldir), woL = fr.toLocal(wo);
                        f3 f   = bsdfEval(bsdf, woL, wiL);
                        if (nonzero(f))
                        {
                            float bp = bsdfPdf(bsdf, woL, wiL, compatPdf);
                            if (GUIDE) bp = gf * bp + guide::mixturePdf(G, ldir);
                            float c  = (DL && compatEsc) ? wiL.z : fabsf(wiL.z);
                            f3    baseV = DL ? value : T * value;
                            float w, pl;
                            if (compatEsc)
                            {
                                w  = misBalanced(lpdf, bp);
                                pl = lpdf;
                            }
                            else
                            {
                                pl = lpdf / float(N);
                                w  = em.type == 1u ? misBalanced(pl, bp) : 1.0f;
                            }
                            Li      = baseV * f;
                            Li      = Li * c;
                            Li      = Li * w;
                            Li      = Li / pl;
                            sdir    = ldir;
                            shadow1 = true;
                        }
                    }
                }
                // BSDF sampling with MIS (raygeneration.cu:391-455 / 234-281).
                float us  = GUIDE ? rng.next1D() : 0.0f;
                f2    u2  = rng.next2D();
                f3    woL = fr.toLocal(wo);
                f3    wiL{0, 0, 0};
                float bp = 0.0f;
                f3    f{0.0f, 0.0f, 0.0f};
                f3    gdir{0.0f, 0.0f, 0.0f};
                if (!GUIDE || us < gf)
                    f = bsdfSample(bsdf, woL, u2, &wiL, &bp);
                else
                {
                    gdir = guide::mixtureSample(G, us - gf, u2.x, u2.y);
                    wiL  = fr.toLocal(gdir);
                    f    = bsdfEval(bsdf, woL, wiL);
                    bp   = bsdfPdf(bsdf, woL, wiL, false);
                }
                const float bpB = bp; // BSDF pdf of the sampled direction (training records)
                if (GUIDE && nonzero(f))
                {
                    if (us < gf) gdir = fr.toWorld(wiL);
                    bp = gf * bp + guide::mixturePdf(G, gdir);
                }
                // The corrected estimator stops paths whose sampled pdf is not
                // positive (0 or NaN at the rim of the cosine warp); the
                // reference's update divides by it (raygeneration.cu:430).
                if (!nonzero(f) || (!compatEsc && !(bp > 0.0f)))
                    finish = true;
                else
                {
                    f3    dir      = GUIDE ? gdir : fr.toWorld(wiL);
                    float lightPdf = sc.hasDome ? domePdf(sc.dome, dir, !compatEsc) : 0.0f;
                    if (DL)
                    {
                        if (sc.hasDome && !(compatEsc && !(lightPdf > 0.0f)))
                        {
                            float c  = compatEsc ? wiL.z : fabsf(wiL.z);
                            float pl = compatEsc ? lightPdf : lightPdf / float(N);
                            Ld       = domeEval(sc.dome, dir, !compatEsc);
                            float w  = misBalanced(bp, pl);
                            f3    kk{f.x * c * w / bp, f.y * c * w / bp, f.z * c * w / bp};
                            Ld      = Ld * kk;
                            sdir2   = dir;
                            shadow2 = true;
                        }
                        finish = true;
                    }
                    else
                    {
                        float c = fabsf(wiL.z);
                        f3    tk{f.x * c / bp, f.y * c / bp, f.z * c / bp};
                        tIn        = T;
                        T          = T * tk;
                        bool alive = true;
                        if (wp.rrStart > 0u && depth >= wp.rrStart)
                        {
                            float q = maxComp(T);
                            q       = q < 1.0f ? q : 1.0f;
                            float r = rng.next1D();
                            if (r >= q)
                                alive = false;
                            else
                                T = T / q;
                        }
                        if (alive)
                        {
                            if (compatEsc)
                            {
                                if (!(lightPdf > 0.0f))
                                    alive = false;
                                else
                                {
                                    float w = misBalanced(bp, lightPdf);
                                    E       = {f.x * c * w / bp, f.y * c * w / bp, f.z * c * w / bp};
                                }
                            }
                            else
                                E = {bp, 0.0f, 0.0f};
                        }
                        if (alive)
                        {
                            pushRay = true;
                            ndir    = dir;
                            info2   = (depth + 1u) | (rng.ctr << 8);
                            if (guided && wp.recStride && slot % wp.recStride == 0u && depth <= P.g.histDepth)
                            {
                                // Training history of this vertex (flushRecords).
                                float4* h = P.g.hist + (size_t(slot / wp.recStride) * P.g.histDepth + depth - 1u) *
                                                           kHistF4;
                                f3 pn = (a.p - f3{P.g.boxMin[0], P.g.boxMin[1], P.g.boxMin[2]}) * P.g.boxScale;
                                h[0]  = make_float4(pn.x, pn.y, pn.z, tIn.x);
                                h[1]  = make_float4(a.ns.x, a.ns.y, a.ns.z, tIn.y);
                                h[2]  = make_float4(wo.x, wo.y, wo.z, tIn.z);
                                h[3]  = make_float4(dir.x, dir.y, dir.z, bpB);
                                h[4]  = make_float4(L.x, L.y, L.z, 0.0f);
                                recBit = 1u << (depth - 1u);
                            }
                        }
                        else
                            finish = true;
                    }
                }
            }
            pushShadow = shadow1 || shadow2;
        }
        // Shadow queue (one entry per path vertex).
        uint32_t sIdx = warpAppend(&P.q.ctr->shadowCount, pushShadow);
        if (pushShadow)
        {
            if (sIdx < P.q.shadowCap)
            {
                uint32_t tag     = slot | (finish ? kLastFlag : 0u);
                P.q.sqO[sIdx]    = make_float4(pHit.x, pHit.y, pHit.z, __uint_as_float(tag));
                P.q.sqD[sIdx]    = make_float4(sdir.x, sdir.y, sdir.z, shadow1 ? 1.0f : 0.0f);
                P.q.sqL[sIdx]    = make_float4(Li.x, Li.y, Li.z, __uint_as_float(vDepth));
                if (DL)
                {
                    P.q.sqD2[sIdx] = make_float4(sdir2.x, sdir2.y, sdir2.z, shadow2 ? 1.0f : 0.0f);
                    P.q.sqL2[sIdx] = make_float4(Ld.x, Ld.y, Ld.z, 0.0f);
                }
            }
            else
                atomicOr(&P.q.ctr->error, 4u);
        }
        // Next-bounce ray queue.
        uint32_t rIdx = warpAppend(&P.q.ctr->rayCount[nxt], pushRay);
        if (pushRay && rIdx >= P.q.slots)
        {
            atomicOr(&P.q.ctr->error, 8u);
            pushRay = false;
        }
        if (pushRay)
        {
            P.q.rqO[nxt][rIdx]    = make_float4(pHit.x, pHit.y, pHit.z, kRayEps);
            P.q.rqD[nxt][rIdx]    = make_float4(ndir.x, ndir.y, ndir.z, FLT_MAX);
            P.q.rqSlot[nxt][rIdx] = slot;
            P.q.psInfo[slot].z    = info2;
            if (GUIDE && recBit) P.q.psInfo[slot].w |= recBit;
            P.q.psT[slot]         = make_float4(T.x, T.y, T.z, 0.0f);
            P.q.psE[slot]         = make_float4(E.x, E.y, E.z, __uint_as_float(cst));
        }
        if (pushRay || (pushShadow && finish)) P.q.psL[slot] = make_float4(L.x, L.y, L.z, 0.0f);
        finishPaths(P, wp, nxt, finish && !pushShadow, slot, L);
    }
}

// Radiance of visible shadow rays, then completion of paths whose last
// vertex had a shadow ray (shadow miss, optix.cu:265-284).
template <bool DL>
__global__ void __launch_bounds__(128) kShadowResolve(Params P, int cur)
{
    const WaveParams wp  = *P.wp;
    const uint32_t   n   = loadCount(&P.q.ctr->shadowCount);
    const int        nxt = cur ^ 1;
    const uint32_t gw = gridDim.x * (blockDim.x >> 5); // static 32-entry batches, as in kShade
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32u; base < n; base += gw * 32u)
    {
        uint32_t i      = base + laneId();
        bool     finish = false;
        uint32_t slot   = 0u;
        f3       L{0, 0, 0};
        if (i < n)
        {
            uint32_t tag = __float_as_uint(P.q.sqO[i].w);
            slot         = tag & ~kLastFlag;
            L            = ld3(P.q.psL[slot]);
            float4 li = P.q.sqL[i];
            if (P.q.vis[DL ? 2 * i : i]) L = L + ld3(li);
            if (DL && P.q.vis[2 * i + 1]) L = L + ld3(P.q.sqL2[i]);
            if (!DL && wp.recStride && slot % wp.recStride == 0u)
            {
                // Guiding: the recorded vertex's radiance snapshot includes
                // its own emitter sample (flushRecords).
                uint32_t d = __float_as_uint(li.w);
                if (d >= 1u && d <= P.g.histDepth && ((P.q.psInfo[slot].w >> (d - 1u)) & 1u))
                    P.g.hist[(size_t(slot / wp.recStride) * P.g.histDepth + d - 1u) * kHistF4 + 4] =
                        make_float4(L.x, L.y, L.z, 0.0f);
            }
            if (tag & kLastFlag)
                finish = true;
            else
                P.q.psL[slot] = make_float4(L.x, L.y, L.z, 0.0f);
        }
        finishPaths(P, wp, nxt, finish, slot, L);
    }
}

// Guided path tracing: network inference after kTraceClosest for the rays of
// the guided shading classes (class queues concatenated in class order), in
// one kernel (kGuideInfer): per 128-row tile, thread t encodes ray k0 + t
// (hit position and shading normal, the 16-level hash-grid gathers, the
// one-blob encodings) straight into the tensor-core A tile, then the tile goes
// through the MLP (cl_mlp_tc.cuh) and each thread writes its ray's lobes.
// The encoding is a chain of dependent gathers (queue -> path state -> hit ->
// vertices -> table); the other CTAs' MMA chains run in its shadow.
constexpr uint32_t kNoRay          = 0xffffffffu;
constexpr int      kGuideEncBlock  = 128;

__device__ __forceinline__ uint32_t guidedCounts(const Params& P, uint32_t* n0, uint32_t* n1)
{
    const uint32_t mask = P.g.classMask;
    *n0                 = (mask & 1u) ? loadCount(&P.q.ctr->classCount[0]) : 0u;
    *n1                 = (mask & 2u) ? loadCount(&P.q.ctr->classCount[1]) : 0u;
    const uint32_t n2   = (mask & 4u) ? loadCount(&P.q.ctr->classCount[2]) : 0u;
    return *n0 + *n1 + n2;
}

// Encoded input row (r: 96 bf16 as 48 pairs) of guided ray k of the
// concatenated class queues; returns its ray-queue index, or kNoRay (and a
// zero row) for a last vertex (depth == maxDepth, not shaded) or a path that
// ends in the radiance cache here.
__device__ __forceinline__ uint32_t encodeGuideRow(const Params& P, const guide::GridView& g, int cur, uint32_t k,
                                                   uint32_t n0, uint32_t n1, uint32_t maxDepth, f3 bmin,
                                                   uint32_t (&r)[guide::kIn / 2], float* in9 = nullptr)
{
    const uint32_t c     = k < n0 ? 0u : (k < n0 + n1 ? 1u : 2u);
    const uint32_t pos   = k - (c == 0u ? 0u : (c == 1u ? n0 : n0 + n1));
    const uint32_t i     = P.q.classIdx[size_t(c) * P.q.slots + pos];
    const uint32_t slot  = P.q.rqSlot[cur][i];
    const uint32_t depth = P.q.psInfo[slot].z & 0xffu;
    if (depth == maxDepth || depth < P.g.minDepth ||
        (P.c.termDepth && depth == P.c.termDepth && !(__float_as_uint(P.q.psE[slot].w) & kCacheTrainBit)))
    {
#pragma unroll
        for (int q = 0; q < guide::kIn / 2; ++q) r[q] = 0u;
        return kNoRay;
    }
    float4  hh = P.q.hit[i];
    float4  rd = P.q.rqD[cur][i];
    HitAttr a  = hitAttributesTri(P.sc, P.q.hitIdx[i], hh.z, hh.w);
    f3      pn = guide::clampUnit((a.p - bmin) * P.g.boxScale);
#pragma unroll
    for (int l = 0; l < guide::kLevels; ++l)
    {
        float2 f = guide::encodeLevel(g, l, pn);
        r[l]     = guide::packBf16(f.x, f.y);
    }
    guide::oneBlobPacked(a.ns, r + guide::kHashF / 2);
    guide::oneBlobPacked(f3{-rd.x, -rd.y, -rd.z}, r + (guide::kHashF + 2 * guide::kBlob) / 2);
    if (in9)
    {
        const float v[9] = {pn.x, pn.y, pn.z, a.ns.x, a.ns.y, a.ns.z, -rd.x, -rd.y, -rd.z};
#pragma unroll
        for (int q = 0; q < 9; ++q) in9[q] = v[q];
    }
    return i;
}

// Radiance cache, first pass: the rays of the surface classes that end
// their path here (depth == termDepth, not a training path) are compacted
// (warp-aggregated append) and encoded like the guide's rows (encodeGuideRow).
__global__ void __launch_bounds__(kGuideEncBlock, 6) kCacheEncode(Params P, guide::GridView g, int cur)
{
    const uint32_t n0 = loadCount(&P.q.ctr->classCount[0]), n1 = loadCount(&P.q.ctr->classCount[1]);
    const uint32_t n  = n0 + n1 + loadCount(&P.q.ctr->classCount[2]);
    const f3       bmin{P.g.boxMin[0], P.g.boxMin[1], P.g.boxMin[2]};
    const uint32_t lane = laneId();
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x)
    {
        const uint32_t k    = base + lane;
        bool           term = false;
        uint32_t       i = 0u, slot = 0u;
        if (k < n)
        {
            const uint32_t c   = k < n0 ? 0u : (k < n0 + n1 ? 1u : 2u);
            const uint32_t pos = k - (c == 0u ? 0u : (c == 1u ? n0 : n0 + n1));
            i                  = P.q.classIdx[size_t(c) * P.q.slots + pos];
            slot               = P.q.rqSlot[cur][i];
            term = (P.q.psInfo[slot].z & 0xffu) == P.c.termDepth && !(__float_as_uint(P.q.psE[slot].w) & kCacheTrainBit);
        }
        const uint32_t idx = warpAppend(&P.q.ctr->cacheCount, term);
        if (!term) continue;
        float4   hh = P.q.hit[i];
        float4   rd = P.q.rqD[cur][i];
        HitAttr  a  = hitAttributesTri(P.sc, P.q.hitIdx[i], hh.z, hh.w);
        f3       pn = guide::clampUnit((a.p - bmin) * P.g.boxScale);
        uint32_t r[guide::kIn / 2];
#pragma unroll
        for (int l = 0; l < guide::kLevels; ++l)
        {
            float2 f = guide::encodeLevel(g, l, pn);
            r[l]     = guide::packBf16(f.x, f.y);
        }
        guide::oneBlobPacked(a.ns, r + guide::kHashF / 2);
        guide::oneBlobPacked(f3{-rd.x, -rd.y, -rd.z}, r + (guide::kHashF + 2 * guide::kBlob) / 2);
        uint4* dst = P.c.enc + size_t(idx) * (guide::kIn / 8);
#pragma unroll
        for (int q = 0; q < guide::kIn / 8; ++q) dst[q] = make_uint4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
        P.c.encIdx[idx] = i;
    }
}

// Guide inference, fused: persistent CTAs of 128 threads; per 128-row tile of
// the guided rays, thread t encodes row t into the tensor-core A tile, the
// tile goes through the MLP (tcgen05, cl_mlp_tc.cuh) and thread t writes the
// head's lobes of its ray, their weights summing to the probability of
// sampling the guide (alpha; < 0: learned).
__global__ void __launch_bounds__(guide::kTcThreads) kGuideInfer(Params P, guide::GridView g, int cur,
                                                                 const uint4* __restrict__ wt, float alpha)
{
    using namespace guide;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t       n0, n1;
    const uint32_t n = guidedCounts(P, &n0, &n1);
    // The grid is fixed (graph replay) while the row count varies by wave:
    // CTAs without a tile skip the weight copy and the TMEM allocation.
    if (blockIdx.x * kTcRows >= n) return;
    const uint32_t tmem     = tcSetup<GuideShape>(smem, wt);
    const uint32_t maxDepth = P.wp->maxDepth;
    const f3       bmin{P.g.boxMin[0], P.g.boxMin[1], P.g.boxMin[2]};
    uint32_t       phase = 0u;
    for (uint32_t k0 = blockIdx.x * kTcRows; k0 < n; k0 += gridDim.x * kTcRows)
    {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t       r[kIn / 2];
        uint32_t       ray = kNoRay;
        float          in9[9];
        const bool     probe = P.g.probe && k < P.g.probeCap;
        if (k < n)
            ray = encodeGuideRow(P, g, cur, k, n0, n1, maxDepth, bmin, r, probe ? in9 : nullptr);
        else
#pragma unroll
            for (int q = 0; q < kIn / 2; ++q) r[q] = 0u;
        const uint32_t vm = __ballot_sync(kFull, ray != kNoRay);
        if (laneId() == 0u && vm) atomicAdd(&P.q.ctr->inferred, (unsigned long long)__popc(vm));
        float o[GuideShape::kOut];
        if (!tcForward<GuideShape>(smem, tmem, r, phase, o))
        {
            if (threadIdx.x == 0) atomicOr(&P.q.ctr->error, kTcTimeout);
            break;
        }
        if (ray != kNoRay)
        {
            Lobes L;
            headLobes(o, &L, alpha);
            float4* dst = P.g.lobes + size_t(ray) * kLobeF4;
#pragma unroll
            for (int j = 0; j < kLobes; ++j) dst[j] = L.l[j];
            dst[8] = make_float4(L.w[0], L.w[1], L.w[2], L.w[3]);
            dst[9] = make_float4(L.w[4], L.w[5], L.w[6], L.w[7]);
            if (probe)
            {
                float* q = P.g.probe + size_t(k) * kProbeF;
#pragma unroll
                for (int j = 0; j < 9; ++j) q[j] = in9[j];
                q[9] = __uint_as_float(ray);
#pragma unroll
                for (int j = 0; j < kLobeF4; ++j)
                {
                    const float4 v = dst[j];
                    q[10 + 4 * j]  = v.x;
                    q[11 + 4 * j]  = v.y;
                    q[12 + 4 * j]  = v.z;
                    q[13 + 4 * j]  = v.w;
                }
            }
        }
        else if (probe)
            P.g.probe[size_t(k) * kProbeF + 9] = __uint_as_float(kNoRay);
    }
    tcTeardown(tmem);
}

// Radiance-cache inference, second pass: persistent CTAs of 128 threads
// stream 128 encoded rows at a time (compacted by kCacheEncode) through the
// MLP on the tensor cores (tcgen05, cl_mlp_tc.cuh), thread t handling row t:
// the predicted radiance per ray, clamped to be non-negative.
__global__ void __launch_bounds__(guide::kTcThreads) kCacheMlp(Params P, const uint4* __restrict__ wt)
{
    using namespace guide;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t n = loadCount(&P.q.ctr->cacheCount);
    if (blockIdx.x * kTcRows >= n) return; // see kGuideInfer
    const uint32_t tmem  = tcSetup<CacheShape>(smem, wt);
    uint32_t       phase = 0u;
    for (uint32_t k0 = blockIdx.x * kTcRows; k0 < n; k0 += gridDim.x * kTcRows)
    {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t       r[kIn / 2];
#pragma unroll
        for (int c = 0; c < kIn / 8; ++c)
        {
            const uint4 v = k < n ? __ldg(P.c.enc + size_t(k) * (kIn / 8) + c) : make_uint4(0u, 0u, 0u, 0u);
            r[4 * c] = v.x, r[4 * c + 1] = v.y, r[4 * c + 2] = v.z, r[4 * c + 3] = v.w;
        }
        const uint32_t ray = k < n ? P.c.encIdx[k] : kNoRay;
        const uint32_t vm  = __ballot_sync(kFull, ray != kNoRay);
        if (laneId() == 0u && vm) atomicAdd(&P.q.ctr->cacheQueries, (unsigned long long)__popc(vm));
        float o[CacheShape::kOut];
        if (!tcForward<CacheShape>(smem, tmem, r, phase, o))
        {
            if (threadIdx.x == 0) atomicOr(&P.q.ctr->error, kTcTimeout);
            break;
        }
        if (ray != kNoRay) P.c.L[ray] = make_float4(fmaxf(o[0], 0.0f), fmaxf(o[1], 0.0f), fmaxf(o[2], 0.0f), 0.0f);
    }
    tcTeardown(tmem);
}
constexpr int kGuideMlpSmem = guide::TcLayout<guide::GuideShape>::kSmem;
constexpr int kCacheMlpSmem = guide::TcLayout<guide::CacheShape>::kSmem;

// CTAs of a tensor-core MLP kernel (guide::kTcThreads threads, `smem` bytes
// of dynamic shared memory) that one SM holds at once: by registers, by
// shared memory (plus the per-CTA reserve) and by TMEM columns (512 per SM,
// guide::kTcCols per CTA).  Counted from the kernel's attributes.
cl_status tcResidentCtas(const void* f, int smem, int* ctas, std::string* err)
{
    cudaFuncAttributes a;
    int                dev = 0, regsSm = 0, smemSm = 0, reserve = 0;
    CL_CUDA(cudaFuncGetAttributes(&a, f), err);
    CL_CUDA(cudaGetDevice(&dev), err);
    CL_CUDA(cudaDeviceGetAttribute(&regsSm, cudaDevAttrMaxRegistersPerMultiprocessor, dev), err);
    CL_CUDA(cudaDeviceGetAttribute(&smemSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev), err);
    CL_CUDA(cudaDeviceGetAttribute(&reserve, cudaDevAttrReservedSharedMemoryPerBlock, dev), err);
    const int warps   = guide::kTcThreads / 32;
    const int regWarp = ((std::max(a.numRegs, 1) + 7) / 8) * 8 * 32; // per-thread count rounded to 8
    const int byRegs  = regsSm / (regWarp * warps);
    const int bySmem  = smemSm / (((smem + int(a.sharedSizeBytes) + reserve + 127) / 128) * 128);
    const int byTmem  = int(512u / guide::kTcCols);
    *ctas             = std::min(std::min(byRegs, bySmem), byTmem);
    if (*ctas < 1)
    {
        *err = "tensor-core MLP pass: no CTA fits on an SM";
        return CL_ERR_STATE;
    }
    return CL_OK;
}

// Records beyond the capacity were dropped; the training step reads the
// clamped count.
__global__ void kClampRecords(Counters* c, uint32_t cap)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) c->trainCount = min(c->recCount, cap);
}
__global__ void kClampCacheRecords(Counters* c, uint32_t cap)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) c->cacheTrainCount = min(c->cacheRec, cap);
}

// Initial fill: slot s starts path s.
__global__ void kRaygen(Params P, uint32_t count)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const WaveParams wp = *P.wp;
    startPath(P, wp, s, s, 0, s);
}

__global__ void kAdvance(Counters* c, int cur)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->raysClosest += c->rayCount[cur];
    c->raysShadow += c->shadowCount;
    c->rayCount[cur] = 0u;
    c->shadowCount   = 0u;
    c->fetchTrace    = 0u;
    c->fetchShadow   = 0u;
    c->fetchInfer    = 0u;
    c->cacheCount    = 0u;
    for (int k = 0; k < 4; ++k)
    {
        c->classCount[k] = 0u;
    }
}

template <bool TWO>
__global__ void __launch_bounds__(kTraceBlock) kOccluded(BvhView bvh, const float4* __restrict__ O,
                                                         const float4* __restrict__ D, uint32_t n,
                                                         uint8_t* __restrict__ occ, uint32_t* err)
{
    extern __shared__ uint2 stack[];
    __shared__ uint8_t      keyLut[kKeyLutBytes];
    fillKeyLut(keyLut);
    uint32_t         i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4        o = O[i], d = D[i];
    float         t, b1, b2;
    TraceCounters tc{0u, 0u};
    uint32_t      h, hi;
    if (TWO)
        h = traverse2<true, false>(bvh, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, o.w, d.w, &t, &b1, &b2, &hi,
                                   stack + threadIdx.x, &tc, err, keyLut);
    else
        h = traverse<true, false>(bvh, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, o.w, d.w, &t, &b1, &b2,
                                  stack + threadIdx.x, &tc, err, keyLut);
    occ[i] = h == kMissPrim ? 0 : 1;
}

__global__ void kAliasSample(DomeView dome, const float2* __restrict__ u, float* dir, float* pdf, float* val, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3    d{0, 0, 0};
    float p = 0.0f;
    float2 uu = u[i];
    f3    v = domeSample(dome, f2{uu.x, uu.y}, true, &d, &p);
    dir[3 * i] = d.x;
    dir[3 * i + 1] = d.y;
    dir[3 * i + 2] = d.z;
    pdf[i] = p;
    val[3 * i] = v.x;
    val[3 * i + 1] = v.y;
    val[3 * i + 2] = v.z;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace
{
using ShadeFn = void (*)(Params, int);

template <bool DL, int MAT> ShadeFn shadeKernelM(uint32_t flags)
{
    uint32_t c   = flags & CL_COMPAT_ALL;
    int      cmp = c == CL_COMPAT_ALL ? 1 : (c == 0u ? 0 : 2);
    bool     al  = (flags & CL_DOME_ALIAS) != 0u;
    if (cmp == 1) return al ? kShade<DL, 1, true, MAT> : kShade<DL, 1, false, MAT>;
    if (cmp == 0) return al ? kShade<DL, 0, true, MAT> : kShade<DL, 0, false, MAT>;
    return al ? kShade<DL, 2, true, MAT> : kShade<DL, 2, false, MAT>;
}

// Guided path-tracing shading of BSDF class MAT (corrected estimator only).
template <int MAT> ShadeFn shadeKernelGuided(uint32_t flags)
{
    return (flags & CL_DOME_ALIAS) ? kShade<false, 0, true, MAT, true> : kShade<false, 0, false, MAT, true>;
}

// Shading kernel of class `mat` (0-2 BSDF type, 3 escaped rays).
template <bool DL> ShadeFn shadeKernelT(int mat, uint32_t flags)
{
    switch (mat)
    {
        case 0: return shadeKernelM<DL, 0>(flags);
        case 1: return shadeKernelM<DL, 1>(flags);
        case 2: return shadeKernelM<DL, 2>(flags);
        default: return shadeKernelM<DL, 3>(flags);
    }
}

ShadeFn shadeKernel(bool dl, int mat, uint32_t flags, bool guided = false)
{
    if (guided && !dl)
    {
        switch (mat)
        {
            case 0: return shadeKernelGuided<0>(flags);
            case 1: return shadeKernelGuided<1>(flags);
            case 2: return shadeKernelGuided<2>(flags);
            default: break;
        }
    }
    return dl ? shadeKernelT<true>(mat, flags) : shadeKernelT<false>(mat, flags);
}
} // namespace

Integrator::Integrator(cl_integrator_type type, uint32_t w, uint32_t h, const cl_render_config& cfg)
    : type_(type), W_(w), H_(h), cfg_(cfg)
{
}

Integrator::~Integrator()
{
    if (graph_) cudaGraphExecDestroy(graph_);
    if (copyStream_) cudaStreamSynchronize(copyStream_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (evResolved_) cudaEventDestroy(evResolved_);
    if (evCopied_) cudaEventDestroy(evCopied_);
    if (copyStream_) cudaStreamDestroy(copyStream_);
    if (evA_) cudaEventDestroy(evA_);
    if (evB_) cudaEventDestroy(evB_);
    for (auto& e : evS_)
        if (e) cudaEventDestroy(e);
    if (hostWp_) cudaFreeHost(hostWp_);
    if (hostCount_) cudaFreeHost(hostCount_);
    if (stream_) cudaStreamDestroy(stream_);
}

cl_status Integrator::init(std::string* err)
{
    if (W_ == 0 || H_ == 0)
    {
        *err = "film size must be non-zero";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg_.max_depth == 0) cfg_.max_depth = 5;
    if (cfg_.max_depth > 255)
    {
        *err = "max_depth must be at most 255";
        return CL_ERR_INVALID_ARG;
    }
    int dev = 0;
    CL_CUDA(cudaGetDevice(&dev), err);
    CL_CUDA(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, dev), err);
    CL_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), err);
    CL_CUDA(cudaStreamCreateWithFlags(&copyStream_, cudaStreamNonBlocking), err);
    CL_CUDA(cudaEventCreateWithFlags(&evResolved_, cudaEventDisableTiming), err);
    CL_CUDA(cudaEventCreateWithFlags(&evCopied_, cudaEventDisableTiming), err);
    CL_CUDA(cudaEventCreate(&evA_), err);
    CL_CUDA(cudaEventCreate(&evB_), err);
    for (auto& e : evS_) CL_CUDA(cudaEventCreate(&e), err);
    CL_CUDA(cudaMallocHost((void**)&hostWp_, sizeof(WaveParams)), err);
    CL_CUDA(cudaMallocHost((void**)&hostCount_, 64), err);
    int b = 0;
    // Occupancy at the deepest supported stack (the launches use less).
    CL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kTraceClosest<false, true>, kTraceBlock,
                                                          traceStackBytes(kStackDepth)),
            err);
    traceBlocks_ = std::max(1, b) * numSMs_;
    CL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kTraceClosest<false, true, true>, kTraceBlock,
                                                          traceStackBytes(kStackDepth)),
            err);
    traceBlocksTwo_ = std::max(1, b) * numSMs_;
    bool dl = type_ == CL_INTEGRATOR_DIRECT_LIGHTING;
    CL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)shadeKernel(dl, 2, cfg_.flags), 128, 0),
            err);
    shadeBlocks_ = std::max(1, b) * numSMs_;
    CL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &b, dl ? (const void*)kShadowResolve<true> : (const void*)kShadowResolve<false>, 128, 0),
            err);
    shadowBlocks_ = std::max(1, b) * numSMs_;
    CL_CUDA(cudaFuncSetAttribute(kGuideInfer, cudaFuncAttributeMaxDynamicSharedMemorySize, kGuideMlpSmem), err);
    CL_CUDA(cudaFuncSetAttribute(kCacheMlp, cudaFuncAttributeMaxDynamicSharedMemorySize, kCacheMlpSmem), err);
    // The whole on-chip memory as shared memory, so that the launch holds the
    // CTAs counted by tcResidentCtas (4 of the guide's and of the cache's).
    CL_CUDA(cudaFuncSetAttribute(kGuideInfer, cudaFuncAttributePreferredSharedMemoryCarveout, 100), err);
    CL_CUDA(cudaFuncSetAttribute(kCacheMlp, cudaFuncAttributePreferredSharedMemoryCarveout, 100), err);
    CL_TRY(tcResidentCtas((const void*)kCacheMlp, kCacheMlpSmem, &b, err));
    cacheMlpBlocks_ = b * numSMs_;
    CL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kCacheEncode, kGuideEncBlock, 0), err);
    cacheEncodeBlocks_ = std::max(1, b) * numSMs_;
    CL_TRY(tcResidentCtas((const void*)kGuideInfer, kGuideMlpSmem, &b, err));
    inferBlocks_ = b * numSMs_;
    CL_TRY(ctr_.alloc(sizeof(Counters), err));
    CL_TRY(wp_.alloc(sizeof(WaveParams), err));
    CL_CUDA(cudaMemsetAsync(ctr_.p, 0, sizeof(Counters), stream_), err);
    return CL_OK;
}

cl_status Integrator::buildMeshes(const cl_mesh_desc* meshes, uint32_t n, std::string* err)
{
    if (!meshes && n)
    {
        *err = "meshes is null";
        return CL_ERR_INVALID_ARG;
    }
    std::vector<HostMesh> out(n);
    for (uint32_t m = 0; m < n; ++m)
    {
        const cl_mesh_desc& d = meshes[m];
        if (!d.positions || !d.indices || !d.tangents || d.num_vertices == 0 || d.num_triangles == 0)
        {
            *err = "mesh " + std::to_string(m) + ": positions, tangents and indices are required";
            return CL_ERR_INVALID_ARG;
        }
        HostMesh& h = out[m];
        size_t    nv = d.num_vertices, nt = d.num_triangles;
        h.pos.assign(d.positions, d.positions + 3 * nv);
        h.tan.assign(d.tangents, d.tangents + 3 * nv);
        h.hasN = d.normals != nullptr;
        if (h.hasN) h.nrm.assign(d.normals, d.normals + 3 * nv);
        h.hasUV = d.uvs != nullptr;
        if (h.hasUV) h.uv.assign(d.uvs, d.uvs + 2 * nv);
        h.idx.assign(d.indices, d.indices + 3 * nt);
        for (uint32_t v : h.idx)
            if (v >= d.num_vertices)
            {
                *err = "mesh " + std::to_string(m) + ": vertex index out of range";
                return CL_ERR_INVALID_ARG;
            }
    }
    meshes_.swap(out);
    sceneBuilt_ = false;
    return CL_OK;
}

// World-space vertices of one instance: 12 floats per vertex {p.xyz, n.xyz,
// t.xyz, u, v, flags}; normals by the inverse transpose of the linear part.
cl_status Integrator::flattenInstance(const HostMesh& m, const float* M, uint32_t i, float* out, std::string* err)
{
    bool ident = M[0] == 1 && M[1] == 0 && M[2] == 0 && M[3] == 0 && M[4] == 0 && M[5] == 1 && M[6] == 0 &&
                 M[7] == 0 && M[8] == 0 && M[9] == 0 && M[10] == 1 && M[11] == 0;
    double a = M[0], b = M[1], c = M[2], d = M[4], e = M[5], f = M[6], g = M[8], h = M[9], k = M[10];
    double det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g);
    if (!ident && std::fabs(det) < 1e-30)
    {
        *err = "instance " + std::to_string(i) + ": singular transform";
        return CL_ERR_INVALID_ARG;
    }
    // Inverse transpose of the linear part, row-major: IT[3 r + c] = inverse[c][r].
    double IT[9] = {(e * k - f * h) / det, -(d * k - f * g) / det, (d * h - e * g) / det,
                    -(b * k - c * h) / det, (a * k - c * g) / det,  -(a * h - b * g) / det,
                    (b * f - c * e) / det,  -(a * f - c * d) / det, (a * e - b * d) / det};
    size_t   mv    = m.pos.size() / 3;
    uint32_t flags = (m.hasN ? 1u : 0u) | (m.hasUV ? 2u : 0u);
    for (size_t v = 0; v < mv; ++v)
    {
        float p[3], nn[3] = {0, 0, 0}, t[3], uv[2] = {0, 0};
        for (int q = 0; q < 3; ++q)
        {
            p[q] = m.pos[3 * v + q];
            t[q] = m.tan[3 * v + q];
            if (m.hasN) nn[q] = m.nrm[3 * v + q];
        }
        if (m.hasUV)
        {
            uv[0] = m.uv[2 * v];
            uv[1] = m.uv[2 * v + 1];
        }
        if (!ident)
        {
            float P2[3], T2[3], N2[3];
            for (int r = 0; r < 3; ++r)
            {
                P2[r] = float(double(M[4 * r]) * p[0] + double(M[4 * r + 1]) * p[1] + double(M[4 * r + 2]) * p[2] +
                              double(M[4 * r + 3]));
                T2[r] = float(double(M[4 * r]) * t[0] + double(M[4 * r + 1]) * t[1] + double(M[4 * r + 2]) * t[2]);
                // n' = (inverse of the linear part)^T n
                N2[r] = float(IT[3 * r] * nn[0] + IT[3 * r + 1] * nn[1] + IT[3 * r + 2] * nn[2]);
            }
            for (int q = 0; q < 3; ++q)
            {
                p[q]  = P2[q];
                t[q]  = T2[q];
                nn[q] = N2[q];
            }
        }
        float* o = out + v * 12;
        o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; o[3] = nn[0];
        o[4] = nn[1]; o[5] = nn[2]; o[6] = t[0]; o[7] = t[1];
        float ff;
        memcpy(&ff, &flags, 4);
        o[8] = t[2]; o[9] = uv[0]; o[10] = uv[1]; o[11] = ff;
    }
    return CL_OK;
}

cl_status Integrator::buildInstances(const cl_instance_desc* inst, uint32_t n, std::string* err)
{
    if ((!inst && n) || n == 0)
    {
        *err = "at least one instance is required";
        return CL_ERR_INVALID_ARG;
    }
    size_t nv = 0, nt = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        if (inst[i].mesh_id >= meshes_.size())
        {
            *err = "instance " + std::to_string(i) + ": mesh_id out of range";
            return CL_ERR_INVALID_ARG;
        }
        nv += meshes_[inst[i].mesh_id].pos.size() / 3;
        nt += meshes_[inst[i].mesh_id].idx.size() / 3;
    }
    if (nt >= 0x7fffffffu || nv >= 0xffffffffu)
    {
        *err = "scene too large";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg_.flags & CL_TWO_LEVEL) return buildTwoLevel(inst, n, err);
    twoLevel_ = false;
    blas_.clear();
    instDev_.release();
    // Flatten instances into world space (the reference's TLAS has no
    // transforms, optix.cu:115; identity transforms are copied exactly).
    std::vector<float>    vtx(nv * 12);
    std::vector<uint32_t> tidx(nt * 4);
    std::vector<float>    tri9(nt * 9);
    std::vector<uint32_t> vtxOff(n);
    size_t vo = 0, to = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        const HostMesh& m = meshes_[inst[i].mesh_id];
        CL_TRY(flattenInstance(m, inst[i].transform, i, &vtx[vo * 12], err));
        vtxOff[i] = uint32_t(vo);
        size_t mv = m.pos.size() / 3;
        size_t mt = m.idx.size() / 3;
        for (size_t t = 0; t < mt; ++t)
        {
            uint32_t* o = &tidx[(to + t) * 4];
            for (int q = 0; q < 3; ++q)
            {
                uint32_t gv = uint32_t(vo + m.idx[3 * t + q]);
                o[q]        = gv;
                for (int c2 = 0; c2 < 3; ++c2) tri9[(to + t) * 9 + 3 * q + c2] = vtx[size_t(gv) * 12 + c2];
            }
            o[3] = inst[i].material_index;
        }
        vo += mv;
        to += mt;
    }
    CL_TRY(vtx_.alloc(vtx.size() * 4, err));
    CL_TRY(triIdx_.alloc(tidx.size() * 4, err));
    CL_TRY(triPos_.alloc(tri9.size() * 4, err));
    CL_CUDA(cudaMemcpyAsync(vtx_.p, vtx.data(), vtx.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaMemcpyAsync(triIdx_.p, tidx.data(), tidx.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaMemcpyAsync(triPos_.p, tri9.data(), tri9.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    // Scene box for the guiding network's position input (uniform scale).
    {
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (size_t v = 0; v < nv; ++v)
            for (int q = 0; q < 3; ++q)
            {
                lo[q] = std::min(lo[q], vtx[v * 12 + q]);
                hi[q] = std::max(hi[q], vtx[v * 12 + q]);
            }
        float ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
        ext       = std::max(ext, 1e-6f) * 1.002f;
        for (int q = 0; q < 3; ++q) boxMin_[q] = lo[q] - 0.001f * ext;
        boxScale_ = 1.0f / ext;
    }
    const auto   w0 = std::chrono::steady_clock::now();
    const double a0 = allocMs();
    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    CL_TRY(buildWideBvh(triPos_.f(), uint32_t(nt), stream_, &bvh_, err));
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    CL_CUDA(cudaEventElapsedTime(&msBvh_, evA_, evB_), err);
    msBvhWall_  = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count());
    msBvhAlloc_ = float(allocMs() - a0);
    triPos_.release();
    CL_TRY(wideBvhSahCost(bvh_, stream_, &sahBuild_, err));
    sah_        = sahBuild_;
    numTris_    = uint32_t(nt);
    sceneBuilt_ = true;
    graphValid_ = false;
    inst_.assign(inst, inst + n);
    instVtxOff_.swap(vtxOff);
    // Material indices are checked at render time against the material count.
    maxMaterialIndex_ = 0;
    for (uint32_t i = 0; i < n; ++i) maxMaterialIndex_ = std::max(maxMaterialIndex_, inst[i].material_index);
    return CL_OK;
}

// Two-level build (CL_TWO_LEVEL): the meshes' object-space vertices and
// triangles in one pool each, one 8-wide BVH per instanced mesh, the instance
// records (transforms, tree pointers, global triangle base in instance
// order, material) and the top tree over the instances' world boxes.  A top
// tree leaf entry is a degenerate "triangle" spanning the instance's box
// (v0 = v2 = min, v1 = max), so the same device builder makes both levels.
static const float kIdentity12[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};

cl_status Integrator::uploadMeshPool(uint32_t meshId, std::string* err)
{
    const HostMesh&    m  = meshes_[meshId];
    const size_t       mv = m.pos.size() / 3;
    std::vector<float> buf(mv * 12);
    CL_TRY(flattenInstance(m, kIdentity12, meshId, buf.data(), err));
    CL_CUDA(cudaMemcpyAsync(vtx_.f() + size_t(meshVtxBase_[meshId]) * 12, buf.data(), buf.size() * 4,
                            cudaMemcpyHostToDevice, stream_),
            err);
    return CL_OK;
}

cl_status Integrator::buildBlas(uint32_t meshId, BuildArena* arena, cudaStream_t st, std::string* err)
{
    const HostMesh&    m  = meshes_[meshId];
    const size_t       mt = m.idx.size() / 3;
    std::vector<float> tri9(mt * 9);
    for (size_t t = 0; t < mt; ++t)
        for (int q = 0; q < 3; ++q)
            for (int c = 0; c < 3; ++c) tri9[t * 9 + 3 * q + c] = m.pos[3 * size_t(m.idx[3 * t + q]) + c];
    BuildArena  local;
    BuildArena& mem = arena ? *arena : local;
    ScratchBuf  d;
    CL_TRY(mem.input(d, tri9.size() * 4, err));
    CL_CUDA(cudaMemcpyAsync(d.p, tri9.data(), tri9.size() * 4, cudaMemcpyHostToDevice, st), err);
    if (!blas_[meshId]) blas_[meshId].reset(new WideBvh());
    return buildWideBvh(d.f(), uint32_t(mt), st, blas_[meshId].get(), err, &mem);
}

// The trees of the instanced meshes.  They are independent, and each build
// waits on the host for its own small launches (cluster counts, collapse
// levels), so up to kBuildThreads host threads build them at once, each on
// its own stream with its own build arena.  Returns after every build ended.
cl_status Integrator::buildBlasAll(const std::vector<uint32_t>& meshes, std::string* err)
{
    constexpr unsigned kBuildThreads = 4;
    const unsigned     nw            = unsigned(std::min<size_t>(kBuildThreads, meshes.size()));
    for (uint32_t m : meshes)
        if (!blas_[m]) blas_[m].reset(new WideBvh());
    if (nw <= 1)
    {
        BuildArena arena;
        for (uint32_t m : meshes) CL_TRY(buildBlas(m, &arena, stream_, err));
        return CL_OK;
    }
    int dev = 0;
    CL_CUDA(cudaGetDevice(&dev), err);
    std::atomic<size_t>      next{0};
    std::atomic<bool>        failed{false};
    std::vector<cl_status>   res(nw, CL_OK);
    std::vector<std::string> msg(nw);
    std::vector<double>      allocs(nw, 0.0);
    std::vector<std::thread> workers;
    for (unsigned w = 0; w < nw; ++w)
        workers.emplace_back([&, w] {
            cudaStream_t s = nullptr;
            if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
            {
                cudaGetLastError();
                res[w] = CL_ERR_CUDA;
                msg[w] = "two-level build: no stream for a build thread";
                failed = true;
                return;
            }
            const double a0 = allocMs();
            {
                BuildArena arena;
                for (size_t k; !failed && (k = next++) < meshes.size();)
                {
                    const cl_status r = buildBlas(meshes[k], &arena, s, &msg[w]);
                    if (r != CL_OK)
                    {
                        res[w] = r;
                        failed = true;
                        break;
                    }
                }
                cudaStreamSynchronize(s); // before the arena's temporaries are freed
            }
            allocs[w] = allocMs() - a0;
            cudaStreamDestroy(s);
        });
    for (auto& t : workers) t.join();
    for (unsigned w = 0; w < nw; ++w) allocMs() += allocs[w];
    for (unsigned w = 0; w < nw; ++w)
        if (res[w] != CL_OK)
        {
            *err = msg[w];
            return res[w];
        }
    return CL_OK;
}

// World box of instance i (every vertex mapped, in double), widened by a
// relative 1e-6 so that FP32 rounding of the object-space traversal cannot
// fall outside it.
void Integrator::instanceBox(uint32_t i, float* lo, float* hi) const
{
    const HostMesh& m  = meshes_[inst_[i].mesh_id];
    const float*    M  = inst_[i].transform;
    double          l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    for (size_t v = 0; v < m.pos.size() / 3; ++v)
        for (int r = 0; r < 3; ++r)
        {
            double x = double(M[4 * r]) * m.pos[3 * v] + double(M[4 * r + 1]) * m.pos[3 * v + 1] +
                       double(M[4 * r + 2]) * m.pos[3 * v + 2] + double(M[4 * r + 3]);
            l[r] = std::min(l[r], x);
            h[r] = std::max(h[r], x);
        }
    double ext = std::max(h[0] - l[0], std::max(h[1] - l[1], h[2] - l[2]));
    for (int r = 0; r < 3; ++r)
    {
        double pad = 1e-6 * ext + 1e-6 * std::max(std::fabs(l[r]), std::fabs(h[r])) + 1e-30;
        lo[r] = float(l[r] - pad);
        hi[r] = float(h[r] + pad);
        if (double(lo[r]) > l[r] - pad) lo[r] = std::nextafter(lo[r], -FLT_MAX);
        if (double(hi[r]) < h[r] + pad) hi[r] = std::nextafter(hi[r], FLT_MAX);
    }
}

cl_status Integrator::buildTopLevel(BuildArena* arena, std::string* err)
{
    const uint32_t     n = uint32_t(inst_.size());
    std::vector<float> tri9(size_t(n) * 9);
    float              slo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, shi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < n; ++i)
    {
        float lo[3], hi[3];
        instanceBox(i, lo, hi);
        for (int c = 0; c < 3; ++c)
        {
            tri9[size_t(i) * 9 + c]     = lo[c];
            tri9[size_t(i) * 9 + 3 + c] = hi[c];
            tri9[size_t(i) * 9 + 6 + c] = lo[c];
            slo[c]                      = std::min(slo[c], lo[c]);
            shi[c]                      = std::max(shi[c], hi[c]);
        }
    }
    // Scene box for the networks' position input (uniform scale).
    float ext = std::max(shi[0] - slo[0], std::max(shi[1] - slo[1], shi[2] - slo[2]));
    ext       = std::max(ext, 1e-6f) * 1.002f;
    for (int q = 0; q < 3; ++q) boxMin_[q] = slo[q] - 0.001f * ext;
    boxScale_ = 1.0f / ext;
    BuildArena  local;
    BuildArena& mem = arena ? *arena : local;
    ScratchBuf  d;
    CL_TRY(mem.input(d, tri9.size() * 4, err));
    CL_CUDA(cudaMemcpyAsync(d.p, tri9.data(), tri9.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    CL_TRY(buildWideBvh(d.f(), n, stream_, &bvh_, err, &mem));
    uint32_t blasDepth = 0;
    for (const auto& b : blas_)
        if (b) blasDepth = std::max(blasDepth, b->depth);
    // Stack: the top tree's pending groups (depth + 1, plus the two entries
    // pushed when a ray enters an instance) and the mesh tree's (depth + 1).
    const uint32_t need = bvh_.depth + 3u + blasDepth + 1u;
    if (need > uint32_t(kStackDepth))
    {
        *err = "two-level scene too deep for the traversal stack (top depth " + std::to_string(bvh_.depth) +
               ", mesh depth " + std::to_string(blasDepth) + ")";
        return CL_ERR_INVALID_ARG;
    }
    twoLevelStack_ = need;
    return CL_OK;
}

cl_status Integrator::uploadInstances(std::string* err)
{
    const uint32_t       n = uint32_t(inst_.size());
    std::vector<InstDev> h(n);
    uint32_t             primBase = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        const float* M = inst_[i].transform;
        const double a = M[0], b = M[1], c = M[2], d = M[4], e = M[5], f = M[6], g = M[8], hh = M[9], k = M[10];
        const double det = a * (e * k - f * hh) - b * (d * k - f * g) + c * (d * hh - e * g);
        if (!(std::fabs(det) > 1e-30))
        {
            *err = "instance " + std::to_string(i) + ": singular transform";
            return CL_ERR_INVALID_ARG;
        }
        // inverse of the linear part, row-major
        const double inv[9] = {(e * k - f * hh) / det, -(b * k - c * hh) / det, (b * f - c * e) / det,
                               -(d * k - f * g) / det, (a * k - c * g) / det,   -(a * f - c * d) / det,
                               (d * hh - e * g) / det, -(a * hh - b * g) / det, (a * e - b * d) / det};
        InstDev& r = h[i];
        for (int row = 0; row < 3; ++row)
        {
            r.o2w[row] = make_float4(M[4 * row], M[4 * row + 1], M[4 * row + 2], M[4 * row + 3]);
            const double tx = -(inv[3 * row] * M[3] + inv[3 * row + 1] * M[7] + inv[3 * row + 2] * M[11]);
            r.w2o[row] = make_float4(float(inv[3 * row]), float(inv[3 * row + 1]), float(inv[3 * row + 2]), float(tx));
        }
        const uint32_t mid = inst_[i].mesh_id;
        r.nodes    = blas_[mid]->nodes.as<const uint4>();
        r.tris     = blas_[mid]->tris.as<const float4>();
        r.primBase = primBase;
        r.triBase  = meshTriBase_[mid];
        r.material = inst_[i].material_index;
        r.flags    = det < 0.0 ? 1u : 0u;
        primBase += uint32_t(meshes_[mid].idx.size() / 3);
    }
    CL_TRY(instDev_.alloc(size_t(n) * sizeof(InstDev), err));
    CL_CUDA(cudaMemcpyAsync(instDev_.p, h.data(), size_t(n) * sizeof(InstDev), cudaMemcpyHostToDevice, stream_), err);
    numTris_ = primBase;
    return CL_OK;
}

cl_status Integrator::buildTwoLevel(const cl_instance_desc* inst, uint32_t n, std::string* err)
{
    // Pools: every mesh's object-space vertices and triangles.
    const uint32_t nm = uint32_t(meshes_.size());
    meshVtxBase_.assign(nm, 0u);
    meshTriBase_.assign(nm, 0u);
    size_t nv = 0, nt = 0;
    for (uint32_t m = 0; m < nm; ++m)
    {
        meshVtxBase_[m] = uint32_t(nv);
        meshTriBase_[m] = uint32_t(nt);
        nv += meshes_[m].pos.size() / 3;
        nt += meshes_[m].idx.size() / 3;
    }
    std::vector<uint32_t> tidx(nt * 4);
    for (uint32_t m = 0; m < nm; ++m)
    {
        const HostMesh& hm = meshes_[m];
        for (size_t t = 0; t < hm.idx.size() / 3; ++t)
        {
            uint32_t* o = &tidx[(meshTriBase_[m] + t) * 4];
            for (int q = 0; q < 3; ++q) o[q] = meshVtxBase_[m] + hm.idx[3 * t + q];
            o[3] = 0u;
        }
    }
    const auto   w0 = std::chrono::steady_clock::now();
    const double a0 = allocMs();
    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    CL_TRY(vtx_.alloc(nv * 48, err));
    CL_TRY(triIdx_.alloc(nt * 16, err));
    CL_CUDA(cudaMemcpyAsync(triIdx_.p, tidx.data(), tidx.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    for (uint32_t m = 0; m < nm; ++m) CL_TRY(uploadMeshPool(m, err));
    std::vector<bool> used(nm, false);
    for (uint32_t i = 0; i < n; ++i) used[inst[i].mesh_id] = true;
    blas_.clear();
    blas_.resize(nm); // null entries
    std::vector<uint32_t> todo;
    for (uint32_t m = 0; m < nm; ++m)
        if (used[m]) todo.push_back(m);
    CL_TRY(buildBlasAll(todo, err));
    inst_.assign(inst, inst + n);
    CL_TRY(buildTopLevel(nullptr, err));
    CL_TRY(uploadInstances(err));
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    CL_CUDA(cudaEventElapsedTime(&msBvh_, evA_, evB_), err);
    msBvhWall_  = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count());
    msBvhAlloc_ = float(allocMs() - a0);
    sahBuild_ = sah_ = 0.0;
    twoLevel_   = true;
    sceneBuilt_ = true;
    graphValid_ = false;
    instVtxOff_.clear();
    maxMaterialIndex_ = 0;
    for (uint32_t i = 0; i < n; ++i) maxMaterialIndex_ = std::max(maxMaterialIndex_, inst[i].material_index);
    return CL_OK;
}

// Vertex edit of a two-level scene: the mesh's pool range is rewritten, its
// tree refitted (CL_BVH_UPDATE_REFIT, _AUTO) or rebuilt (_REBUILD), and the
// top tree rebuilt over the instances' new boxes.
cl_status Integrator::updateTwoLevel(uint32_t meshId, uint32_t mode, std::string* err)
{
    CL_TRY(uploadMeshPool(meshId, err));
    float ms = 0.0f;
    msBvhRefit_ = 0.0f;
    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    if (blas_[meshId])
    {
        if (mode == CL_BVH_UPDATE_REBUILD)
        {
            CL_TRY(buildBlas(meshId, nullptr, stream_, err));
            ++rebuilds_;
        }
        else
        {
            CL_TRY(refitWideBvh(blas_[meshId].get(), vtx_.p, triIdx_.as<uint4>() + meshTriBase_[meshId], stream_, err));
            ++refits_;
        }
    }
    CL_TRY(buildTopLevel(nullptr, err));
    CL_TRY(uploadInstances(err));
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    CL_CUDA(cudaEventElapsedTime(&ms, evA_, evB_), err);
    msBvhUpdate_ = ms;
    graphValid_  = false;
    return resetIteration(err);
}

cl_status Integrator::updateMeshVertices(uint32_t meshId, const float* pos, const float* nrm, const float* tan,
                                         uint32_t count, uint32_t mode, std::string* err)
{
    if (!sceneBuilt_)
    {
        *err = "no scene: build meshes and instances first";
        return CL_ERR_STATE;
    }
    if (meshId >= meshes_.size())
    {
        *err = "mesh_id out of range";
        return CL_ERR_INVALID_ARG;
    }
    HostMesh& m = meshes_[meshId];
    if (!pos || size_t(count) * 3 != m.pos.size())
    {
        *err = "positions are required, with the mesh's vertex count (" + std::to_string(m.pos.size() / 3) + ")";
        return CL_ERR_INVALID_ARG;
    }
    if (mode > CL_BVH_UPDATE_REBUILD)
    {
        *err = "unknown BVH update mode";
        return CL_ERR_INVALID_ARG;
    }
    for (size_t i = 0; i < size_t(count) * 3; ++i)
        if (!std::isfinite(pos[i]))
        {
            *err = "vertex " + std::to_string(i / 3) + ": position is not finite";
            return CL_ERR_INVALID_ARG;
        }
    m.pos.assign(pos, pos + size_t(count) * 3);
    if (nrm)
    {
        m.nrm.assign(nrm, nrm + size_t(count) * 3);
        m.hasN = true;
    }
    if (tan) m.tan.assign(tan, tan + size_t(count) * 3);
    if (twoLevel_) return updateTwoLevel(meshId, mode, err);

    // Re-flatten the instances of this mesh into their vertex ranges.
    std::vector<float> buf;
    for (size_t i = 0; i < inst_.size(); ++i)
    {
        if (inst_[i].mesh_id != meshId) continue;
        buf.resize(size_t(count) * 12);
        CL_TRY(flattenInstance(m, inst_[i].transform, uint32_t(i), buf.data(), err));
        CL_CUDA(cudaMemcpyAsync(vtx_.f() + size_t(instVtxOff_[i]) * 12, buf.data(), buf.size() * 4,
                                cudaMemcpyHostToDevice, stream_),
                err);
    }

    // Device time of the refit and/or rebuild (the surface-area cost pass
    // and the vertex upload are not included).
    bool  rebuild = mode == CL_BVH_UPDATE_REBUILD;
    float ms      = 0.0f;
    msBvhRefit_   = 0.0f;
    if (!rebuild)
    {
        CL_CUDA(cudaEventRecord(evA_, stream_), err);
        CL_TRY(refitWideBvh(&bvh_, vtx_.p, triIdx_.p, stream_, err));
        CL_CUDA(cudaEventRecord(evB_, stream_), err);
        CL_CUDA(cudaEventSynchronize(evB_), err);
        CL_CUDA(cudaEventElapsedTime(&ms, evA_, evB_), err);
        msBvhRefit_ = ms;
        CL_TRY(wideBvhSahCost(bvh_, stream_, &sah_, err));
        ++refits_;
        // A refit keeps the topology: once the moved geometry has made the
        // tree much costlier than a fresh build, rebuild.
        rebuild = mode == CL_BVH_UPDATE_AUTO && sah_ > kRefitSahLimit * sahBuild_;
    }
    if (rebuild)
    {
        float        msBuild = 0.0f;
        const auto   w0      = std::chrono::steady_clock::now();
        const double a0      = allocMs();
        CL_CUDA(cudaEventRecord(evA_, stream_), err);
        CL_TRY(triPos_.alloc(size_t(numTris_) * 36, err));
        CL_TRY(gatherTrianglePositions(vtx_.p, triIdx_.p, numTris_, triPos_.f(), stream_, err));
        cl_status st = buildWideBvh(triPos_.f(), numTris_, stream_, &bvh_, err);
        triPos_.release();
        if (st != CL_OK)
        {
            sceneBuilt_ = false;
            return st;
        }
        CL_CUDA(cudaEventRecord(evB_, stream_), err);
        CL_CUDA(cudaEventSynchronize(evB_), err);
        CL_CUDA(cudaEventElapsedTime(&msBuild, evA_, evB_), err);
        ms += msBuild;
        msBvh_      = msBuild;
        msBvhWall_  = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count());
        msBvhAlloc_ = float(allocMs() - a0);
        CL_TRY(wideBvhSahCost(bvh_, stream_, &sahBuild_, err));
        sah_        = sahBuild_;
        graphValid_ = false; // new node and triangle buffers
        ++rebuilds_;
    }
    msBvhUpdate_ = ms;
    // RenderEngine::compileAccelStructs (renderengine.cpp:65-77): a shape
    // edit restarts progressive accumulation.
    return resetIteration(err);
}

cl_status Integrator::buildMaterials(const cl_material_desc* m, uint32_t n, std::string* err)
{
    if (!m || n == 0)
    {
        *err = "at least one material is required";
        return CL_ERR_INVALID_ARG;
    }
    std::vector<float> h(size_t(n) * 4 * kMatF4);
    uint32_t           maxTex = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        const cl_material_desc& d = m[i];
        if (d.type > CL_MATERIAL_GLASS)
        {
            *err = "material " + std::to_string(i) + ": unknown type";
            return CL_ERR_INVALID_ARG;
        }
        // GlassMtl has no textures (glass.h:17-27); DiffuseMtl no roughness.
        if ((d.type == CL_MATERIAL_GLASS && (d.reflectance_texture || d.roughness_texture)) ||
            (d.type == CL_MATERIAL_DIFFUSE && d.roughness_texture))
        {
            *err = "material " + std::to_string(i) + ": this type takes no such texture";
            return CL_ERR_INVALID_ARG;
        }
        uint32_t refs[3] = {d.reflectance_texture, d.roughness_texture, d.normal_texture};
        for (uint32_t r : refs)
        {
            if (r > textures_.size())
            {
                *err = "material " + std::to_string(i) + ": texture " + std::to_string(r) + " (1-based) of " +
                       std::to_string(textures_.size()) + " built";
                return CL_ERR_INVALID_ARG;
            }
            maxTex = std::max(maxTex, r);
        }
        if (d.type == CL_MATERIAL_GLASS && d.interior_ior == 1.0f)
        {
            *err = "material " + std::to_string(i) + ": glass IOR must differ from 1 (roughdielectric.h:28)";
            return CL_ERR_INVALID_ARG;
        }
        float*   o = &h[size_t(i) * 4 * kMatF4];
        uint32_t t = d.type;
        memcpy(&o[0], &t, 4);
        memcpy(&o[12], refs, 12);
        o[15] = 0.0f;
        o[1]  = d.reflectance[0];
        o[2]  = d.reflectance[1];
        o[3]  = d.reflectance[2];
        o[4]  = d.roughness * d.roughness; // metal.h:52, glass.h:26
        o[5]  = d.interior_ior;
        o[6]  = d.eta[0];
        o[7]  = d.eta[1];
        o[8]  = d.eta[2];
        o[9]  = d.k[0];
        o[10] = d.k[1];
        o[11] = d.k[2];
    }
    CL_TRY(mats_.alloc(h.size() * 4, err));
    CL_CUDA(cudaMemcpyAsync(mats_.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    numMaterials_  = n;
    maxTextureRef_ = maxTex;
    graphValid_    = false;
    return CL_OK;
}

cl_status Integrator::buildTextures(const cl_texture_desc* t, uint32_t n, std::string* err)
{
    graphValid_ = false;
    return textures_.build(t, n, stream_, err);
}

cl_status Integrator::buildEmitters(const cl_emitter_desc* e, uint32_t n, std::string* err)
{
    if ((!e && n) || n > uint32_t(kMaxEmitters))
    {
        *err = "between 0 and 8 emitters are supported";
        return CL_ERR_INVALID_ARG;
    }
    std::vector<EmitterDev> out;
    int                     domeIdx = -1;
    for (uint32_t i = 0; i < n; ++i)
    {
        EmitterDev d{};
        d.type = e[i].type;
        if (e[i].type == CL_EMITTER_DIRECTIONAL)
            d.dl = DirectionalLight{{e[i].intensity[0], e[i].intensity[1], e[i].intensity[2]},
                                    {e[i].direction[0], e[i].direction[1], e[i].direction[2]},
                                    e[i].angular_radius};
        else if (e[i].type == CL_EMITTER_HDRI_DOME)
        {
            if (!e[i].texels || e[i].width == 0 || e[i].height == 0)
            {
                *err = "dome emitter needs texels and a size";
                return CL_ERR_INVALID_ARG;
            }
            domeIdx = int(i);
        }
        else
        {
            *err = "emitter " + std::to_string(i) + ": unknown type";
            return CL_ERR_INVALID_ARG;
        }
        out.push_back(d);
    }
    hasDome_ = false;
    if (domeIdx >= 0)
    {
        CL_CUDA(cudaEventRecord(evA_, stream_), err);
        CL_TRY(buildDome(e[domeIdx].texels, int(e[domeIdx].width), int(e[domeIdx].height), stream_, &dome_, err));
        CL_CUDA(cudaEventRecord(evB_, stream_), err);
        CL_CUDA(cudaEventSynchronize(evB_), err);
        CL_CUDA(cudaEventElapsedTime(&msDome_, evA_, evB_), err);
        hasDome_ = true;
    }
    emitters_.swap(out);
    graphValid_ = false;
    return CL_OK;
}

cl_status Integrator::updateCamera(const cl_camera* c, std::string* err)
{
    if (!c)
    {
        *err = "camera is null";
        return CL_ERR_INVALID_ARG;
    }
    if (!hasCamera_ || memcmp(&camera_, c, sizeof(cl_camera)) != 0)
    {
        camera_    = *c;
        hasCamera_ = true;
        return resetIteration(err); // path.h:73-80
    }
    return CL_OK;
}

cl_status Integrator::ensureFilm(std::string* err)
{
    size_t np = size_t(W_) * H_;
    if (!film_.p || film_.bytes != np * 16)
    {
        graphValid_ = false;
        CL_TRY(film_.alloc(np * 16, err));
        CL_CUDA(cudaMemsetAsync(film_.p, 0, np * 16, stream_), err);
    }
    if ((cfg_.flags & CL_FILM_FP64) && (!film64_.p || film64_.bytes != np * 48))
    {
        graphValid_ = false;
        CL_TRY(film64_.alloc(np * 48, err));
        CL_CUDA(cudaMemsetAsync(film64_.p, 0, np * 48, stream_), err);
    }
    return CL_OK;
}

cl_status Integrator::clearFilm(std::string* err)
{
    if (film_.p) CL_CUDA(cudaMemsetAsync(film_.p, 0, film_.bytes, stream_), err);
    if (film64_.p) CL_CUDA(cudaMemsetAsync(film64_.p, 0, film64_.bytes, stream_), err);
    filmSpp_ = 0;
    return CL_OK;
}

cl_status Integrator::ensureQueues(std::string* err)
{
    uint32_t slots = cfg_.path_slots ? cfg_.path_slots : (1u << 21);
    if (slots > kMaxPathSlots)
    {
        *err = "path_slots " + std::to_string(slots) + " above the maximum " + std::to_string(kMaxPathSlots);
        return CL_ERR_INVALID_ARG;
    }
    if (slots == slots_ && rqO_[0].p) return CL_OK;
    size_t s = slots;
    for (int q = 0; q < 2; ++q)
    {
        CL_TRY(rqO_[q].alloc(s * 16, err));
        CL_TRY(rqD_[q].alloc(s * 16, err));
        CL_TRY(rqSlot_[q].alloc(s * 4, err));
    }
    CL_TRY(hit_.alloc(s * 16, err));
    CL_TRY(hitIdx_.alloc(s * 16, err));
    CL_TRY(hitInst_.alloc(s * 4, err));
    CL_TRY(sqO_.alloc(s * 16, err));
    CL_TRY(sqD_.alloc(s * 16, err));
    CL_TRY(sqL_.alloc(s * 16, err));
    if (type_ == CL_INTEGRATOR_DIRECT_LIGHTING)
    {
        CL_TRY(sqD2_.alloc(s * 16, err));
        CL_TRY(sqL2_.alloc(s * 16, err));
    }
    CL_TRY(vis_.alloc(s * 2, err));
    CL_TRY(classIdx_.alloc(s * 4 * 4, err));
    CL_TRY(psInfo_.alloc(s * 16, err));
    CL_TRY(psT_.alloc(s * 16, err));
    CL_TRY(psE_.alloc(s * 16, err));
    CL_TRY(psL_.alloc(s * 16, err));
    slots_      = slots;
    shadowCap_  = slots;
    graphValid_ = false;
    return CL_OK;
}

BvhView Integrator::bvhView() const
{
    // Named members (not an aggregate list): the struct's field order is no
    // part of this function's contract.
    BvhView v{};
    v.nodes = bvh_.nodes.as<const uint4>();
    v.tris  = bvh_.tris.as<const float4>();
    if (twoLevel_)
    {
        v.inst       = instDev_.as<const InstDev>();
        v.stackDepth = twoLevelStack_;
        return v;
    }
    v.inst       = nullptr;
    v.stackDepth = std::min<uint32_t>(bvh_.depth + 1u, uint32_t(kStackDepth));
    return v;
}

ClassifyView Integrator::classifyView() const
{
    return ClassifyView{triIdx_.as<const uint4>(), mats_.as<const float4>(), classIdx_.u(), slots_, hitIdx_.as<uint4>(),
                        hitInst_.u()};
}

Params Integrator::params() const
{
    Params P{};
    P.sc.bvh       = bvhView();
    P.sc.triIdx    = triIdx_.as<const uint4>();
    P.sc.vtx       = vtx_.as<const float4>();
    P.sc.mats      = mats_.as<const float4>();
    P.sc.tex       = textures_.device();
    P.sc.hasDome   = hasDome_ ? 1 : 0;
    if (hasDome_) P.sc.dome = dome_.view();
    P.sc.numEmitters = uint32_t(emitters_.size());
    for (size_t i = 0; i < emitters_.size(); ++i) P.sc.emitters[i] = emitters_[i];
    for (int q = 0; q < 2; ++q)
    {
        P.q.rqO[q]    = rqO_[q].as<float4>();
        P.q.rqD[q]    = rqD_[q].as<float4>();
        P.q.rqSlot[q] = rqSlot_[q].u();
    }
    P.q.hit       = hit_.as<float4>();
    P.q.hitIdx    = hitIdx_.as<const uint4>();
    P.q.sqO       = sqO_.as<float4>();
    P.q.sqD       = sqD_.as<float4>();
    P.q.sqL       = sqL_.as<float4>();
    P.q.sqD2      = sqD2_.as<float4>();
    P.q.sqL2      = sqL2_.as<float4>();
    P.q.vis       = vis_.as<uint8_t>();
    P.q.classIdx  = classIdx_.u();
    P.q.psInfo    = psInfo_.as<uint4>();
    P.q.psT       = psT_.as<float4>();
    P.q.psE       = psE_.as<float4>();
    P.q.psL       = psL_.as<float4>();
    P.q.film      = film_.as<float4>();
    P.q.film64    = (cfg_.flags & CL_FILM_FP64) ? film64_.as<double>() : nullptr;
    P.q.ctr       = ctr_.as<Counters>();
    P.q.slots     = slots_;
    P.q.shadowCap = shadowCap_;
    P.wp          = wp_.as<const WaveParams>();
    if (guide_)
    {
        P.g.lobes     = lobes_.as<float4>();
        P.g.hist      = hist_.as<float4>();
        P.g.rec       = rec_.as<float4>();
        P.g.recCap    = recCap_;
        P.g.classMask = guideCfg_.class_mask;
        P.g.minDepth  = std::max(guideCfg_.min_depth, 1u);
        P.g.minAlpha  = guideCfg_.min_alpha;
        P.g.histDepth = histDepth_;
    }
    for (int q = 0; q < 3; ++q) P.g.boxMin[q] = boxMin_[q];
    P.g.boxScale = boxScale_;
    if (cache_)
    {
        P.c.L         = cacheL_.as<float4>();
        P.c.enc       = cacheEnc_.as<uint4>();
        P.c.encIdx    = cacheEncIdx_.u();
        P.c.hist      = cacheHist_.as<float4>();
        P.c.rec       = cacheRec_.as<float4>();
        P.c.recCap    = cacheRecCap_;
        P.c.termDepth = cacheCfg_.prefix_bounces + 1u;
        P.c.trainMask = (1u << cacheCfg_.train_log2_fraction) - 1u;
        P.c.histDepth = cacheHistDepth_;
    }
    return P;
}

cl_status Integrator::launchWave(int cur, bool profile, std::string* err)
{
    Params P  = params();
    bool   dl = type_ == CL_INTEGRATOR_DIRECT_LIGHTING;
    Counters* c = ctr_.as<Counters>();
    const bool st = cfg_.flags & CL_TRACE_STATS;
    if (profile) CL_CUDA(cudaEventRecord(evS_[0], stream_), err);
    {
        const size_t sb = traceStackBytes(P.sc.bvh.stackDepth);
        auto         k  = st ? (twoLevel_ ? kTraceClosest<true, true, true> : kTraceClosest<true, true, false>)
                             : (twoLevel_ ? kTraceClosest<false, true, true> : kTraceClosest<false, true, false>);
        k<<<tBlocks(), kTraceBlock, sb, stream_>>>(P.sc.bvh, P.q.rqO[cur], P.q.rqD[cur], &c->rayCount[cur],
                                                      &c->fetchTrace, P.q.hit, c, classifyView());
        if (profile) CL_CUDA(cudaEventRecord(evS_[5], stream_), err);
        (twoLevel_ ? kClassifyHits<true> : kClassifyHits<false>)<<<numSMs_ * 8, kClassifyThreads, 0, stream_>>>(
            P.sc.bvh, P.q.hit, &c->rayCount[cur], c, classifyView());
    }
    if (profile) CL_CUDA(cudaEventRecord(evS_[1], stream_), err);
    const uint32_t gmask = guide_ ? guideCfg_.class_mask : 0u;
    if (gmask)
    {
        kGuideInfer<<<inferBlocks_, guide::kTcThreads, kGuideMlpSmem, stream_>>>(
            P, guide_->grid(), cur, guide_->tcWeights(),
            guideCfg_.learn_selection ? -1.0f : 1.0f - guideCfg_.bsdf_fraction);
    }
    if (cache_)
    {
        kCacheEncode<<<cacheEncodeBlocks_, kGuideEncBlock, 0, stream_>>>(P, cache_->grid(), cur);
        kCacheMlp<<<cacheMlpBlocks_, guide::kTcThreads, kCacheMlpSmem, stream_>>>(P, cache_->tcWeights());
    }
    if (profile) CL_CUDA(cudaEventRecord(evS_[4], stream_), err);
    for (int m = 0; m < 4; ++m)
        shadeKernel(dl, m, cfg_.flags, m < 3 && ((gmask >> m) & 1u))<<<shadeBlocks_, 128, 0, stream_>>>(P, cur);
    if (profile) CL_CUDA(cudaEventRecord(evS_[2], stream_), err);
    {
        using ShadowFn = void (*)(Params);
        const ShadowFn table[2][2][2] = {
            {{kTraceShadow<false, false, false>, kTraceShadow<false, false, true>},
             {kTraceShadow<false, true, false>, kTraceShadow<false, true, true>}},
            {{kTraceShadow<true, false, false>, kTraceShadow<true, false, true>},
             {kTraceShadow<true, true, false>, kTraceShadow<true, true, true>}}};
        table[dl][st][twoLevel_]<<<tBlocks(), kTraceBlock, traceStackBytes(P.sc.bvh.stackDepth), stream_>>>(P);
    }
    if (dl)
        kShadowResolve<true><<<shadowBlocks_, 128, 0, stream_>>>(P, cur);
    else
        kShadowResolve<false><<<shadowBlocks_, 128, 0, stream_>>>(P, cur);
    if (profile) CL_CUDA(cudaEventRecord(evS_[3], stream_), err);
    kAdvance<<<1, 32, 0, stream_>>>(c, cur);
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

cl_status Integrator::captureGraph(std::string* err)
{
    if (graph_)
    {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    cudaGraph_t g = nullptr;
    CL_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), err);
    cl_status s = CL_OK;
    for (int w = 0; w < 4 && s == CL_OK; ++w) s = launchWave(w & 1, false, err);
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (s != CL_OK) return s;
    CL_CUDA(e, err);
    CL_CUDA(cudaGraphInstantiate(&graph_, g, 0), err);
    cudaGraphDestroy(g);
    graphValid_ = true;
    return CL_OK;
}

cl_status Integrator::render(uint32_t spp, std::string* err)
{
    if (!sceneBuilt_ || !mats_.p || !hasCamera_)
    {
        *err = "render needs meshes, instances, materials and a camera";
        return CL_ERR_STATE;
    }
    if (maxMaterialIndex_ >= numMaterials_)
    {
        *err = "an instance references material " + std::to_string(maxMaterialIndex_) + " of " +
               std::to_string(numMaterials_);
        return CL_ERR_INVALID_ARG;
    }
    if (maxTextureRef_ > textures_.size())
    {
        *err = "a material references texture " + std::to_string(maxTextureRef_) + " (1-based) of " +
               std::to_string(textures_.size());
        return CL_ERR_STATE;
    }
    if (spp == 0) return CL_OK;
    if (guide_ || cache_) CL_TRY(refuseIfTcSuspect(err));
    CL_TRY(ensureFilm(err));
    CL_TRY(ensureQueues(err));
    msRender_ = msTrace_ = msShade_ = msShadow_ = msInfer_ = 0.0f;
    waves_ = 0;
    waveRays_.clear();
    lastRaysC_ = lastRaysS_ = lastNodes_ = lastTris_ = lastNodesS_ = lastTrisS_ = 0;
    if (guide_) CL_TRY(ensureGuideBuffers(err));
    if (cache_) CL_TRY(ensureCacheBuffers(err));
    // Online training: one step per network on the records of each sample
    // per pixel while a network trains (the guide for its first train_spp
    // spp; the cache for its first train_spp spp, or for every spp when 0),
    // then the remaining samples in one pass.
    for (;;)
    {
        const bool tg = guide_ && guide_->steps() < guideCfg_.train_spp;
        const bool tc = cache_ && (cacheCfg_.train_spp == 0u || cache_->steps() < cacheCfg_.train_spp);
        if (spp == 0 || (!tg && !tc)) break;
        CL_TRY(renderPass(1, tg, tc, err));
        --spp;
        if (tg) CL_TRY(trainGuide(err));
        if (tc) CL_TRY(trainCache(err));
    }
    if (spp > 0) CL_TRY(renderPass(spp, false, false, err));
    return CL_OK;
}

cl_status Integrator::trainGuide(std::string* err)
{
    Counters* dc = ctr_.as<Counters>();
    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    kClampRecords<<<1, 32, 0, stream_>>>(dc, recCap_);
    CL_CUDA(cudaGetLastError(), err);
    CL_TRY(guide_->trainDevice(rec_.as<const float4>(), &dc->trainCount, err));
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    CL_CUDA(cudaMemcpyAsync(hostCount_, &dc->recCount, 8, cudaMemcpyDeviceToHost, stream_), err);
    double loss = 0.0;
    CL_CUDA(cudaMemcpyAsync(&loss, guide_->lossDev(), 8, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    CL_TRY(guide_->checkTrainErr(err));
    float t = 0.0f;
    CL_CUDA(cudaEventElapsedTime(&t, evA_, evB_), err);
    msTrain_ += t;
    msRender_ += t;
    guideRecordsLast_ = hostCount_[0];
    guideSamples_ += std::min(hostCount_[1], guideCfg_.batch);
    guideLoss_ = loss;
    return CL_OK;
}

cl_status Integrator::trainCache(std::string* err)
{
    Counters* dc = ctr_.as<Counters>();
    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    kClampCacheRecords<<<1, 32, 0, stream_>>>(dc, cacheRecCap_);
    CL_CUDA(cudaGetLastError(), err);
    CL_TRY(cache_->trainDevice(cacheRec_.as<const float4>(), &dc->cacheTrainCount, err));
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    CL_CUDA(cudaMemcpyAsync(hostCount_ + 2, &dc->cacheRec, 8, cudaMemcpyDeviceToHost, stream_), err);
    double loss = 0.0;
    CL_CUDA(cudaMemcpyAsync(&loss, cache_->lossDev(), 8, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    CL_TRY(cache_->checkTrainErr(err));
    float t = 0.0f;
    CL_CUDA(cudaEventElapsedTime(&t, evA_, evB_), err);
    msCacheTrain_ += t;
    msRender_ += t;
    cacheRecordsLast_ = hostCount_[2];
    cacheSamples_ += std::min(hostCount_[3], cacheCfg_.network.batch);
    cacheLoss_ = loss;
    return CL_OK;
}

cl_status Integrator::beginPass(uint32_t spp, bool record, bool cacheTrain, uint32_t* initSlots, std::string* err)
{
    const bool  dl = type_ == CL_INTEGRATOR_DIRECT_LIGHTING;
    WaveParams& wp = *hostWp_;
    wp.W           = W_;
    wp.H           = H_;
    wp.frame0      = iteration_;
    wp.maxDepth    = dl ? 1u : cfg_.max_depth;
    wp.rrStart     = cfg_.rr_start_depth;
    wp.flags       = cfg_.flags;
    wp.dl          = dl ? 1u : 0u;
    wp.recStride   = record ? recStride_ : 0u;
    wp.cacheTrain  = cacheTrain ? 1u : 0u;
    wp.totalPaths  = (unsigned long long)W_ * H_ * spp;
    memcpy(wp.cam, &camera_, sizeof(camera_));
    CL_CUDA(cudaMemcpyAsync(wp_.p, hostWp_, sizeof(WaveParams), cudaMemcpyHostToDevice, stream_), err);
    uint32_t init = uint32_t(std::min<unsigned long long>(slots_, wp.totalPaths));
    Counters c0{};
    c0.rayCount[0] = init;
    c0.pathNext    = init;
    CL_CUDA(cudaMemcpyAsync(ctr_.p, &c0, sizeof(Counters), cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err); // hostWp_/c0 reused next call
    waveRaysSeen_ = 0ull;
    *initSlots    = init;
    return CL_OK;
}

cl_status Integrator::renderPass(uint32_t spp, bool record, bool cacheTrain, std::string* err)
{
    const bool profile = cfg_.flags & CL_PROFILE_STAGES;
    uint32_t   init    = 0u;
    CL_TRY(beginPass(spp, record, cacheTrain, &init, err));
    const WaveParams& wp = *hostWp_;

    CL_CUDA(cudaEventRecord(evA_, stream_), err);
    kRaygen<<<(init + 255) / 256, 256, 0, stream_>>>(params(), init);
    CL_CUDA(cudaGetLastError(), err);
    if (!profile && !graphValid_) CL_TRY(captureGraph(err));

    Counters* dc = ctr_.as<Counters>();
    // Every path needs at most maxDepth waves and at least one path per slot
    // finishes per maxDepth waves, so this bound is never reached by a
    // correct schedule.
    const unsigned long long maxIter =
        ((unsigned long long)(wp.maxDepth + 1) * (wp.totalPaths / slots_ + 2) + 16) / 4 + 1;
    for (unsigned long long iter = 0;; ++iter)
    {
        if (iter >= maxIter)
        {
            *err = "render did not drain its queues";
            return CL_ERR_TIMEOUT;
        }
        if (profile)
        {
            for (int w = 0; w < 4; ++w)
            {
                CL_TRY(launchWave(w & 1, true, err));
                unsigned long long rc = 0ull;
                CL_CUDA(cudaMemcpyAsync(&rc, &dc->raysClosest, 8, cudaMemcpyDeviceToHost, stream_), err);
                CL_CUDA(cudaStreamSynchronize(stream_), err);
                waveRays_.push_back(rc - waveRaysSeen_);
                waveRaysSeen_ = rc;
                float a = 0, b = 0, c = 0, d = 0, e = 0;
                CL_CUDA(cudaEventElapsedTime(&a, evS_[0], evS_[5]), err);
                CL_CUDA(cudaEventElapsedTime(&e, evS_[5], evS_[1]), err);
                CL_CUDA(cudaEventElapsedTime(&d, evS_[1], evS_[4]), err);
                CL_CUDA(cudaEventElapsedTime(&b, evS_[4], evS_[2]), err);
                CL_CUDA(cudaEventElapsedTime(&c, evS_[2], evS_[3]), err);
                msTrace_ += a;
                msInfer_ += d;
                msShade_ += b + e;
                msShadow_ += c;
            }
        }
        else
            CL_CUDA(cudaGraphLaunch(graph_, stream_), err);
        waves_ += 4;
        CL_CUDA(cudaMemcpyAsync(hostCount_, &dc->rayCount[0], 4, cudaMemcpyDeviceToHost, stream_), err);
        CL_CUDA(cudaStreamSynchronize(stream_), err);
        if (hostCount_[0] == 0u) break;
    }
    CL_CUDA(cudaEventRecord(evB_, stream_), err);
    Counters ch;
    CL_CUDA(cudaMemcpyAsync(&ch, ctr_.p, sizeof(Counters), cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaEventSynchronize(evB_), err);
    float msPass = 0.0f;
    CL_CUDA(cudaEventElapsedTime(&msPass, evA_, evB_), err);
    msRender_ += msPass;
    if (ch.error)
    {
        *err = std::string("device error flags ") + std::to_string(ch.error) +
               (ch.error & 1u ? " (traversal stack overflow)" : "") + (ch.error & 4u ? " (shadow queue overflow)" : "") +
               (ch.error & 8u ? " (ray queue overflow)" : "") +
               (ch.error & guide::kTcTimeout ? " (tensor-core wait ran out)" : "");
        if (ch.error & guide::kTcTimeout)
        {
            markTcSuspect();
            return CL_ERR_TIMEOUT;
        }
        return (ch.error & 12u) ? CL_ERR_QUEUE_OVERFLOW : CL_ERR_STATE;
    }
    pathsDone_ += wp.totalPaths;
    raysClosest_ += ch.raysClosest;
    raysShadow_ += ch.raysShadow;
    lastRaysC_ += ch.raysClosest;
    lastRaysS_ += ch.raysShadow;
    lastNodes_ += ch.statNodes;
    lastTris_ += ch.statTris;
    lastNodesS_ += ch.statNodesS;
    lastTrisS_ += ch.statTrisS;
    guideInferred_ += ch.inferred;
    cacheQueries_ += ch.cacheQueries;
    launches_ = waves_;
    iteration_ += spp;
    filmSpp_ += spp;
    return CL_OK;
}

cl_status Integrator::ensureGuideBuffers(std::string* err)
{
    const uint64_t wh    = uint64_t(W_) * H_;
    const uint32_t batch = guideCfg_.batch;
    recStride_           = uint32_t(std::max<uint64_t>(1, wh / batch));
    histSlots_           = (slots_ + recStride_ - 1) / recStride_;
    histDepth_           = std::min(cfg_.max_depth, 32u);
    recCap_              = uint32_t(std::min<uint64_t>(4ull * batch, 1ull << 26));
    const size_t lb = size_t(slots_) * kLobeF4 * 16, hb = size_t(histSlots_) * histDepth_ * kHistF4 * 16,
                 rb = size_t(recCap_) * kRecordF4 * 16;
    if (lobes_.bytes != lb)
    {
        CL_TRY(lobes_.alloc(lb, err));
        graphValid_ = false;
    }
    if (hist_.bytes != hb)
    {
        CL_TRY(hist_.alloc(hb, err));
        graphValid_ = false;
    }
    if (rec_.bytes != rb)
    {
        CL_TRY(rec_.alloc(rb, err));
        graphValid_ = false;
    }
    return CL_OK;
}

cl_status Integrator::setGuiding(const cl_guide_config* cfg, std::string* err)
{
    if (!cfg)
    {
        guide_.reset();
        lobes_.release();
        hist_.release();
        rec_.release();
        graphValid_ = false;
        return resetIteration(err);
    }
    if (type_ != CL_INTEGRATOR_PATH_TRACING)
    {
        *err = "guiding needs the path-tracing integrator";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg_.flags & CL_COMPAT_ALL)
    {
        *err = "guiding needs the corrected estimator (no CL_COMPAT_* flag)";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg->class_mask & ~7u)
    {
        *err = "guide class_mask has bits beyond the three BSDF classes";
        return CL_ERR_INVALID_ARG;
    }
    std::unique_ptr<GuideNet> g(new GuideNet(*cfg));
    CL_TRY(g->init(stream_, err));
    guide_    = std::move(g);
    guideCfg_ = *cfg;
    guideSamples_ = guideRecordsLast_ = guideInferred_ = 0;
    guideLoss_ = 0.0;
    msTrain_ = msInfer_ = 0.0f;
    graphValid_ = false;
    return resetIteration(err);
}

cl_status Integrator::guideStats(cl_guide_stats* s, std::string* err) const
{
    if (!guide_)
    {
        *err = "guiding is off";
        return CL_ERR_STATE;
    }
    s->steps           = guide_->steps();
    s->samples_trained = guideSamples_;
    s->records_last    = guideRecordsLast_;
    s->inferred        = guideInferred_;
    s->last_loss       = guideLoss_;
    s->ms_train        = msTrain_;
    s->ms_infer        = msInfer_;
    return CL_OK;
}

cl_status Integrator::ensureCacheBuffers(std::string* err)
{
    cacheHistDepth_ = std::min(cfg_.max_depth, 31u);
    cacheRecCap_    = uint32_t(std::min<uint64_t>(4ull * cacheCfg_.network.batch, 1ull << 26));
    const size_t lb = size_t(slots_) * 16, eb = size_t(slots_) * guide::kIn * 2,
                 hb = size_t(slots_) * cacheHistDepth_ * kCacheHistF4 * 16, rb = size_t(cacheRecCap_) * kRecordF4 * 16;
    if (cacheL_.bytes != lb)
    {
        CL_TRY(cacheL_.alloc(lb, err));
        CL_TRY(cacheEncIdx_.alloc(size_t(slots_) * 4, err));
        graphValid_ = false;
    }
    if (cacheEnc_.bytes != eb)
    {
        CL_TRY(cacheEnc_.alloc(eb, err));
        graphValid_ = false;
    }
    if (cacheHist_.bytes != hb)
    {
        CL_TRY(cacheHist_.alloc(hb, err));
        graphValid_ = false;
    }
    if (cacheRec_.bytes != rb)
    {
        CL_TRY(cacheRec_.alloc(rb, err));
        graphValid_ = false;
    }
    return CL_OK;
}

cl_status Integrator::setRadianceCache(const cl_radiance_cache_config* cfg, std::string* err)
{
    if (!cfg)
    {
        cache_.reset();
        cacheL_.release();
        cacheEnc_.release();
        cacheEncIdx_.release();
        cacheHist_.release();
        cacheRec_.release();
        graphValid_ = false;
        return resetIteration(err);
    }
    if (type_ != CL_INTEGRATOR_PATH_TRACING)
    {
        *err = "the radiance cache needs the path-tracing integrator";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg_.flags & CL_COMPAT_ALL)
    {
        *err = "the radiance cache needs the corrected estimator (no CL_COMPAT_* flag)";
        return CL_ERR_INVALID_ARG;
    }
    if (cfg->prefix_bounces < 1u || cfg->prefix_bounces > 254u || cfg->train_log2_fraction > 16u)
    {
        *err = "radiance cache: prefix_bounces must be in [1, 254], train_log2_fraction in [0, 16]";
        return CL_ERR_INVALID_ARG;
    }
    std::unique_ptr<CacheNet> c(new CacheNet(cfg->network));
    CL_TRY(c->init(stream_, err));
    cache_    = std::move(c);
    cacheCfg_ = *cfg;
    cacheSamples_ = cacheRecordsLast_ = cacheQueries_ = 0;
    cacheLoss_    = 0.0;
    msCacheTrain_ = 0.0f;
    graphValid_   = false;
    return resetIteration(err);
}

cl_status Integrator::cacheStats(cl_guide_stats* s, std::string* err) const
{
    if (!cache_)
    {
        *err = "the radiance cache is off";
        return CL_ERR_STATE;
    }
    s->steps           = cache_->steps();
    s->samples_trained = cacheSamples_;
    s->records_last    = cacheRecordsLast_;
    s->inferred        = cacheQueries_;
    s->last_loss       = cacheLoss_;
    s->ms_train        = msCacheTrain_;
    s->ms_infer        = 0.0f;
    return CL_OK;
}

// Mean radiance of the film into the staging buffer (alpha 1).
__global__ void kResolveFilm(const float4* __restrict__ film, float4* __restrict__ out, uint32_t n, float inv)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float4 f = film[i];
        out[i]   = make_float4(f.x * inv, f.y * inv, f.z * inv, 1.0f);
    }
}

cl_status Integrator::resolveFilm(std::string* err)
{
    size_t np = size_t(W_) * H_;
    CL_TRY(ensureFilm(err));
    if (resolve_.bytes != np * 16)
    {
        CL_CUDA(cudaStreamSynchronize(copyStream_), err); // no copy may still read the old buffer
        CL_TRY(resolve_.alloc(np * 16, err));
    }
    // The staging buffer is reused: the previous copy out of it must be done.
    CL_CUDA(cudaStreamWaitEvent(stream_, evCopied_, 0), err);
    float inv = filmSpp_ ? 1.0f / float(filmSpp_) : 0.0f;
    kResolveFilm<<<numSMs_ * 4, 256, 0, stream_>>>(film_.as<const float4>(), resolve_.as<float4>(), uint32_t(np), inv);
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

cl_status Integrator::readbackFilm(float* rgba, size_t bytes, std::string* err)
{
    size_t np = size_t(W_) * H_;
    if (!rgba || bytes < np * 16)
    {
        *err = "film buffer too small";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(resolveFilm(err));
    CL_CUDA(cudaMemcpyAsync(rgba, resolve_.p, np * 16, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    return CL_OK;
}

cl_status Integrator::readbackFilmAsync(float* rgba, size_t bytes, std::string* err)
{
    size_t np = size_t(W_) * H_;
    if (!rgba || bytes < np * 16)
    {
        *err = "film buffer too small";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(resolveFilm(err));
    CL_CUDA(cudaEventRecord(evResolved_, stream_), err);
    CL_CUDA(cudaStreamWaitEvent(copyStream_, evResolved_, 0), err);
    CL_CUDA(cudaMemcpyAsync(rgba, resolve_.p, np * 16, cudaMemcpyDeviceToHost, copyStream_), err);
    CL_CUDA(cudaEventRecord(evCopied_, copyStream_), err);
    return CL_OK;
}

cl_status Integrator::readbackWait(std::string* err)
{
    CL_CUDA(cudaEventSynchronize(evCopied_), err);
    return CL_OK;
}

cl_status Integrator::readbackFilmStats(double* sum, double* sumsq, size_t count, std::string* err)
{
    size_t np = size_t(W_) * H_;
    if (!(cfg_.flags & CL_FILM_FP64))
    {
        *err = "FP64 film not enabled (CL_FILM_FP64)";
        return CL_ERR_STATE;
    }
    if (!sum || !sumsq || count < np * 3)
    {
        *err = "film stats buffers too small";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(ensureFilm(err));
    std::vector<double> h(np * 6);
    CL_CUDA(cudaMemcpyAsync(h.data(), film64_.p, np * 48, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    for (size_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c)
        {
            sum[3 * i + c]   = h[6 * i + c];
            sumsq[3 * i + c] = h[6 * i + 3 + c];
        }
    return CL_OK;
}

cl_status Integrator::resize(uint32_t w, uint32_t h, std::string* err)
{
    if (w == 0 || h == 0)
    {
        *err = "film size must be non-zero";
        return CL_ERR_INVALID_ARG;
    }
    W_ = w;
    H_ = h;
    film_.release();
    film64_.release();
    CL_TRY(ensureFilm(err));
    iteration_ = 0;
    filmSpp_   = 0;
    return CL_OK;
}

cl_status Integrator::resetIteration(std::string* err) { return setIteration(0u, err); }

cl_status Integrator::setIteration(uint32_t iteration, std::string* err)
{
    iteration_ = iteration;
    return clearFilm(err);
}

void Integrator::stats(cl_stats* s) const
{
    memset(s, 0, sizeof(*s));
    s->paths          = pathsDone_;
    s->rays_closest   = raysClosest_;
    s->rays_shadow    = raysShadow_;
    s->iteration      = iteration_;
    s->spp            = filmSpp_;
    s->bvh_nodes      = bvh_.numNodes;
    s->bvh_depth      = bvh_.depth;
    s->triangles      = numTris_;
    s->waves          = waves_;
    s->ms_bvh_build   = msBvh_;
    s->ms_dome_build  = msDome_;
    s->ms_last_render = msRender_;
    s->ms_trace       = msTrace_;
    s->ms_shade       = msShade_;
    s->ms_shadow      = msShadow_;
    s->launches       = launches_;
    s->trace_nodes    = lastNodes_;
    s->trace_tris     = lastTris_;
    s->shadow_nodes   = lastNodesS_;
    s->shadow_tris    = lastTrisS_;
    s->last_rays_closest = lastRaysC_;
    s->last_rays_shadow  = lastRaysS_;
    s->ms_bvh_update     = msBvhUpdate_;
    s->ms_bvh_build_wall  = msBvhWall_;
    s->ms_bvh_build_alloc = msBvhAlloc_;
    s->ms_bvh_refit      = msBvhRefit_;
    s->bvh_refits        = refits_;
    s->bvh_rebuilds      = rebuilds_;
    s->bvh_sah           = sah_;
    s->bvh_sah_build     = sahBuild_;
}

cl_status Integrator::getBvh(void* nodes, size_t nodeBytes, void* tris, size_t triBytes, std::string* err)
{
    if (!sceneBuilt_)
    {
        *err = "no scene";
        return CL_ERR_STATE;
    }
    size_t nb = size_t(bvh_.numNodes) * 80, tb = size_t(bvh_.numTris) * 48;
    if ((nodes && nodeBytes < nb) || (tris && triBytes < tb))
    {
        *err = "buffer too small: nodes need " + std::to_string(nb) + " bytes, triangles " + std::to_string(tb);
        return CL_ERR_INVALID_ARG;
    }
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    if (nodes) CL_CUDA(cudaMemcpy(nodes, bvh_.nodes.p, nb, cudaMemcpyDeviceToHost), err);
    if (tris) CL_CUDA(cudaMemcpy(tris, bvh_.tris.p, tb, cudaMemcpyDeviceToHost), err);
    return CL_OK;
}

cl_status Integrator::traceRays(const float* rays, uint32_t n, float* t, uint32_t* prim, float* b1, float* b2,
                                std::string* err)
{
    if (!sceneBuilt_)
    {
        *err = "scene not built";
        return CL_ERR_STATE;
    }
    if (n == 0) return CL_OK;
    if (!rays || !t || !prim || !b1 || !b2)
    {
        *err = "null argument";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(ensureQueues(err));
    std::vector<float4> o(slots_), d(slots_), h(slots_);
    Counters* dc = ctr_.as<Counters>();
    for (uint32_t base = 0; base < n; base += slots_)
    {
        uint32_t m = std::min(slots_, n - base);
        for (uint32_t i = 0; i < m; ++i)
        {
            const float* r = rays + 8 * size_t(base + i);
            o[i]           = make_float4(r[0], r[1], r[2], r[3]);
            d[i]           = make_float4(r[4], r[5], r[6], r[7]);
        }
        CL_CUDA(cudaMemcpyAsync(rqO_[0].p, o.data(), m * 16, cudaMemcpyHostToDevice, stream_), err);
        CL_CUDA(cudaMemcpyAsync(rqD_[0].p, d.data(), m * 16, cudaMemcpyHostToDevice, stream_), err);
        Counters c0{};
        c0.rayCount[0] = m;
        CL_CUDA(cudaMemcpyAsync(ctr_.p, &c0, sizeof(c0), cudaMemcpyHostToDevice, stream_), err);
        (twoLevel_ ? kTraceClosest<false, false, true> : kTraceClosest<false, false, false>)
            <<<tBlocks(), kTraceBlock, traceStackBytes(bvhView().stackDepth), stream_>>>(
                bvhView(), rqO_[0].as<float4>(), rqD_[0].as<float4>(), &dc->rayCount[0], &dc->fetchTrace,
                hit_.as<float4>(), dc, ClassifyView{});
        CL_CUDA(cudaGetLastError(), err);
        CL_CUDA(cudaMemcpyAsync(h.data(), hit_.p, m * 16, cudaMemcpyDeviceToHost, stream_), err);
        Counters ch;
        CL_CUDA(cudaMemcpyAsync(&ch, ctr_.p, sizeof(ch), cudaMemcpyDeviceToHost, stream_), err);
        CL_CUDA(cudaStreamSynchronize(stream_), err);
        if (ch.error)
        {
            *err = "traversal error flags " + std::to_string(ch.error);
            return CL_ERR_STATE;
        }
        for (uint32_t i = 0; i < m; ++i)
        {
            t[base + i]    = h[i].x;
            uint32_t pb;
            memcpy(&pb, &h[i].y, 4);
            prim[base + i] = pb;
            b1[base + i]   = h[i].z;
            b2[base + i]   = h[i].w;
        }
    }
    return CL_OK;
}

cl_status Integrator::occludedRays(const float* rays, uint32_t n, uint8_t* occ, std::string* err)
{
    if (!sceneBuilt_)
    {
        *err = "scene not built";
        return CL_ERR_STATE;
    }
    if (n == 0) return CL_OK;
    if (!rays || !occ)
    {
        *err = "null argument";
        return CL_ERR_INVALID_ARG;
    }
    DevBuf o, d, r;
    CL_TRY(o.alloc(size_t(n) * 16, err));
    CL_TRY(d.alloc(size_t(n) * 16, err));
    CL_TRY(r.alloc(n, err));
    std::vector<float4> ho(n), hd(n);
    for (uint32_t i = 0; i < n; ++i)
    {
        const float* q = rays + 8 * size_t(i);
        ho[i]          = make_float4(q[0], q[1], q[2], q[3]);
        hd[i]          = make_float4(q[4], q[5], q[6], q[7]);
    }
    CL_CUDA(cudaMemcpyAsync(o.p, ho.data(), size_t(n) * 16, cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaMemcpyAsync(d.p, hd.data(), size_t(n) * 16, cudaMemcpyHostToDevice, stream_), err);
    CL_CUDA(cudaMemsetAsync(ctr_.p, 0, sizeof(Counters), stream_), err);
    (twoLevel_ ? kOccluded<true> : kOccluded<false>)
        <<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, traceStackBytes(bvhView().stackDepth), stream_>>>(
        bvhView(), o.as<float4>(), d.as<float4>(), n,
        r.as<uint8_t>(), &ctr_.as<Counters>()->error);
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemcpyAsync(occ, r.p, n, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    return CL_OK;
}

cl_status Integrator::traceStats(const float* rays, uint32_t n, uint64_t* nodes, uint64_t* tris, std::string* err)
{
    if (!sceneBuilt_)
    {
        *err = "scene not built";
        return CL_ERR_STATE;
    }
    if (!rays || !nodes || !tris)
    {
        *err = "null argument";
        return CL_ERR_INVALID_ARG;
    }
    CL_TRY(ensureQueues(err));
    Counters* dc = ctr_.as<Counters>();
    uint64_t  an = 0, at = 0;
    std::vector<float4> o(slots_), d(slots_);
    for (uint32_t base = 0; base < n; base += slots_)
    {
        uint32_t m = std::min(slots_, n - base);
        for (uint32_t i = 0; i < m; ++i)
        {
            const float* r = rays + 8 * size_t(base + i);
            o[i]           = make_float4(r[0], r[1], r[2], r[3]);
            d[i]           = make_float4(r[4], r[5], r[6], r[7]);
        }
        CL_CUDA(cudaMemcpyAsync(rqO_[0].p, o.data(), m * 16, cudaMemcpyHostToDevice, stream_), err);
        CL_CUDA(cudaMemcpyAsync(rqD_[0].p, d.data(), m * 16, cudaMemcpyHostToDevice, stream_), err);
        Counters c0{};
        c0.rayCount[0] = m;
        CL_CUDA(cudaMemcpyAsync(ctr_.p, &c0, sizeof(c0), cudaMemcpyHostToDevice, stream_), err);
        (twoLevel_ ? kTraceClosest<true, false, true> : kTraceClosest<true, false, false>)
            <<<tBlocks(), kTraceBlock, traceStackBytes(bvhView().stackDepth), stream_>>>(
                bvhView(), rqO_[0].as<float4>(), rqD_[0].as<float4>(), &dc->rayCount[0], &dc->fetchTrace,
                hit_.as<float4>(), dc, ClassifyView{});
        CL_CUDA(cudaGetLastError(), err);
        Counters ch;
        CL_CUDA(cudaMemcpyAsync(&ch, ctr_.p, sizeof(ch), cudaMemcpyDeviceToHost, stream_), err);
        CL_CUDA(cudaStreamSynchronize(stream_), err);
        an += ch.statNodes;
        at += ch.statTris;
    }
    *nodes = an;
    *tris  = at;
    return CL_OK;
}

cl_status Integrator::domeTables(float* pU, float* cU, float* pV, float* cV, std::string* err)
{
    if (!hasDome_)
    {
        *err = "no dome emitter";
        return CL_ERR_STATE;
    }
    size_t a = size_t(dome_.w + 1) * dome_.h * 4, b = size_t(dome_.h + 1) * 4;
    if (pU) CL_CUDA(cudaMemcpyAsync(pU, dome_.pU.p, a, cudaMemcpyDeviceToHost, stream_), err);
    if (cU) CL_CUDA(cudaMemcpyAsync(cU, dome_.cU.p, a, cudaMemcpyDeviceToHost, stream_), err);
    if (pV) CL_CUDA(cudaMemcpyAsync(pV, dome_.pV.p, b, cudaMemcpyDeviceToHost, stream_), err);
    if (cV) CL_CUDA(cudaMemcpyAsync(cV, dome_.cV.p, b, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    return CL_OK;
}

// Test probe of the fused guide inference: the first wave of the next
// frame (camera rays), traced and run through kGuideInfer exactly as in a
// render, with each guided row's network input (position in the scene box,
// shading normal, outgoing direction), ray index and lobes copied out.  No
// shading runs, so the film is untouched; the iteration index is kept.
cl_status Integrator::guideProbe(uint32_t cap, float* rows, uint32_t* count, std::string* err)
{
    if (!rows || !count)
    {
        *err = "guide probe: null output";
        return CL_ERR_INVALID_ARG;
    }
    if (!guide_ || !guideCfg_.class_mask)
    {
        *err = "guide probe: guiding is off";
        return CL_ERR_STATE;
    }
    if (!sceneBuilt_ || !mats_.p || !hasCamera_)
    {
        *err = "guide probe needs a built scene and a camera";
        return CL_ERR_STATE;
    }
    CL_TRY(refuseIfTcSuspect(err));
    CL_TRY(ensureFilm(err));
    CL_TRY(ensureQueues(err));
    CL_TRY(ensureGuideBuffers(err));
    DevBuf probe;
    CL_TRY(probe.alloc(size_t(std::max(cap, 1u)) * kProbeF * 4, err));
    uint32_t init = 0u;
    CL_TRY(beginPass(1, false, false, &init, err));
    Params P       = params();
    P.g.probe      = probe.f();
    P.g.probeCap   = cap;
    Counters* c    = ctr_.as<Counters>();
    kRaygen<<<(init + 255) / 256, 256, 0, stream_>>>(P, init);
    (twoLevel_ ? kTraceClosest<false, true, true> : kTraceClosest<false, true, false>)
        <<<tBlocks(), kTraceBlock, traceStackBytes(P.sc.bvh.stackDepth), stream_>>>(
            P.sc.bvh, P.q.rqO[0], P.q.rqD[0], &c->rayCount[0], &c->fetchTrace, P.q.hit, c, classifyView());
    (twoLevel_ ? kClassifyHits<true> : kClassifyHits<false>)<<<numSMs_ * 8, kClassifyThreads, 0, stream_>>>(
        P.sc.bvh, P.q.hit, &c->rayCount[0], c, classifyView());
    kGuideInfer<<<inferBlocks_, guide::kTcThreads, kGuideMlpSmem, stream_>>>(
        P, guide_->grid(), 0, guide_->tcWeights(), guideCfg_.learn_selection ? -1.0f : 1.0f - guideCfg_.bsdf_fraction);
    CL_CUDA(cudaGetLastError(), err);
    Counters ch;
    CL_CUDA(cudaMemcpyAsync(&ch, ctr_.p, sizeof(Counters), cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    if (ch.error)
    {
        if (ch.error & guide::kTcTimeout) markTcSuspect();
        *err = "guide probe: device error flags " + std::to_string(ch.error);
        return (ch.error & guide::kTcTimeout) ? CL_ERR_TIMEOUT : CL_ERR_STATE;
    }
    uint32_t n = 0u;
    for (int m = 0; m < 3; ++m)
        if ((guideCfg_.class_mask >> m) & 1u) n += ch.classCount[m];
    n      = std::min(n, cap);
    *count = n;
    if (n) CL_CUDA(cudaMemcpy(rows, probe.p, size_t(n) * kProbeF * 4, cudaMemcpyDeviceToHost), err);
    return CL_OK;
}

cl_status Integrator::waveRays(uint64_t* out, uint32_t cap, uint32_t* count, std::string* err) const
{
    if (!count || (!out && cap))
    {
        *err = "null argument";
        return CL_ERR_INVALID_ARG;
    }
    const uint32_t n = uint32_t(std::min<size_t>(cap, waveRays_.size()));
    for (uint32_t i = 0; i < n; ++i) out[i] = waveRays_[i];
    *count = uint32_t(waveRays_.size());
    return CL_OK;
}

cl_status Integrator::domeAliasTables(uint32_t* aliasRow, uint32_t* aliasCol, std::string* err)
{
    if (!hasDome_)
    {
        *err = "no dome emitter";
        return CL_ERR_STATE;
    }
    if (aliasRow)
        CL_CUDA(cudaMemcpyAsync(aliasRow, dome_.aliasRow.p, size_t(dome_.h) * 8, cudaMemcpyDeviceToHost, stream_), err);
    if (aliasCol)
        CL_CUDA(cudaMemcpyAsync(aliasCol, dome_.aliasCol.p, size_t(dome_.w) * dome_.h * 8, cudaMemcpyDeviceToHost,
                                stream_),
                err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    return CL_OK;
}

cl_status Integrator::domeAliasSample(const float* u2, float* dir, float* pdf, float* val, uint32_t n, std::string* err)
{
    if (!hasDome_)
    {
        *err = "no dome emitter";
        return CL_ERR_STATE;
    }
    if (n == 0) return CL_OK;
    DevBuf du, dd, dp, dv;
    CL_TRY(du.alloc(size_t(n) * 8, err));
    CL_TRY(dd.alloc(size_t(n) * 12, err));
    CL_TRY(dp.alloc(size_t(n) * 4, err));
    CL_TRY(dv.alloc(size_t(n) * 12, err));
    CL_CUDA(cudaMemcpyAsync(du.p, u2, size_t(n) * 8, cudaMemcpyHostToDevice, stream_), err);
    kAliasSample<<<(n + 255) / 256, 256, 0, stream_>>>(dome_.view(), du.as<float2>(), dd.f(), dp.f(), dv.f(), n);
    CL_CUDA(cudaGetLastError(), err);
    CL_CUDA(cudaMemcpyAsync(dir, dd.p, size_t(n) * 12, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaMemcpyAsync(pdf, dp.p, size_t(n) * 4, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaMemcpyAsync(val, dv.p, size_t(n) * 12, cudaMemcpyDeviceToHost, stream_), err);
    CL_CUDA(cudaStreamSynchronize(stream_), err);
    return CL_OK;
}

} // namespace clb
