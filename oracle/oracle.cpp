// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's wavefront integrators, one path at a
// time, plus a binned-SAH binary BVH and a brute-force intersector that give
// the exact closest hit under the shared watertight ray-triangle test.
//
//   * Path tracing: WavefrontPathTracingIntegrator::render
//     (src/core/integrators/path.cpp:84-231) with the kernels
//     generateCameraRays (src/kernel/integrators/raygeneration.cu:59-103),
//     evaluateEscapedRays (:105-136), evaluateMaterialsAndLightsPathTracing
//     (:285-456), the OptiX programs (src/core/devices/optix.cu:38-284) and
//     LightSampler::sampleEmitterDirect (libkernel/base/emitter.h:168-202).
//   * Direct lighting: WavefrontDirectLightingIntegrator::render
//     (src/core/integrators/direct.cpp:84-201) with
//     evaluateMaterialsAndLightsDirectLighting (raygeneration.cu:139-282).
//
// A path's random numbers depend only on (pixel, frame, counter)
// (sampler.h:45-55), so tracing path by path gives the same per-sample
// values as the reference's queue order.  The film is the per-sample path
// radiance summed in FP64 (sum and sum of squares per pixel); the reference's
// running-mean + sRGB round trip (quirk Q8) is not reproduced by either build.
//
// Flags (kCompat*) select the reference's behaviour (compat) or the corrected
// estimator; Russian roulette is new in both builds (absent from the reference,
// path.cpp:135) and identical here and on the GPU.

#include "orc_emit.h"

#include <atomic>
#include <cfloat>
#include <cstdio>
#include <memory>
#include <thread>
#include <array>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace
{
// ---------------------------------------------------------------------------
// Binary BVH, binned SAH (16 bins), leaves of at most 4 triangles.  Boxes are
// widened by a relative 2^-20 so that the box test never culls a triangle the
// watertight test accepts; the triangle test alone decides hits.
// ---------------------------------------------------------------------------
struct Box
{
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void  grow(const float* p)
    {
        for (int i = 0; i < 3; ++i)
        {
            lo[i] = std::min(lo[i], p[i]);
            hi[i] = std::max(hi[i], p[i]);
        }
    }
    void grow(const Box& b)
    {
        for (int i = 0; i < 3; ++i)
        {
            lo[i] = std::min(lo[i], b.lo[i]);
            hi[i] = std::max(hi[i], b.hi[i]);
        }
    }
    float area() const
    {
        float d[3];
        for (int i = 0; i < 3; ++i) d[i] = std::max(0.0f, hi[i] - lo[i]);
        return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct Node
{
    Box      box;
    uint32_t left = 0, count = 0, first = 0; // leaf if count > 0
};

struct Scene
{
    // geometry
    std::vector<float>    tri;    // 9 floats per triangle (world positions)
    std::vector<uint32_t> order;  // leaf order -> triangle id
    std::vector<Node>     nodes;
    MeshView              mesh{};
    const uint32_t*       triMaterial = nullptr;
    uint32_t              ntris       = 0;
    // materials: constants and 1-based texture indices {reflectance, roughness, normal map}
    std::vector<Bsdf<float>>               materials;
    std::vector<std::array<uint32_t, 3>>   matTex;
    std::vector<Texture>                   textures;
    // emitters: in list order (light-selection order), plus the dome
    struct Em
    {
        int         type; // 0 directional, 1 dome
        Directional dir;
    };
    std::vector<Em>    emitters;
    bool               hasDome = false;
    Dome               dome;
    std::vector<float> domeTex, pU, cU, pV, cV;
    std::vector<uint32_t> aliasRow, aliasCol; // set by orc_scene_set_dome_tables
    // camera
    V3<float> camPos{}, d00{}, ddu{}, ddv{};
};

struct BuildItem
{
    Box   b;
    float c[3];
};

void buildRec(Scene& s, std::vector<BuildItem>& items, std::vector<uint32_t>& ids, uint32_t begin, uint32_t end,
              uint32_t nodeIdx, std::atomic<uint32_t>& nodeCount, int depth)
{
    Node& node = s.nodes[nodeIdx];
    Box   bb, cb;
    for (uint32_t i = begin; i < end; ++i)
    {
        bb.grow(items[ids[i]].b);
        cb.grow(items[ids[i]].c);
    }
    node.box        = bb;
    uint32_t n      = end - begin;
    auto     makeLeaf = [&]() {
        node.first = begin;
        node.count = n;
    };
    if (n <= 4 || depth > 60)
    {
        makeLeaf();
        return;
    }
    constexpr int B    = 16;
    float         best = FLT_MAX;
    int           bestAxis = -1, bestSplit = -1;
    for (int axis = 0; axis < 3; ++axis)
    {
        float ext = cb.hi[axis] - cb.lo[axis];
        if (!(ext > 0.0f)) continue;
        Box      bins[B];
        uint32_t cnt[B] = {};
        float    scale  = float(B) / ext;
        for (uint32_t i = begin; i < end; ++i)
        {
            const BuildItem& it = items[ids[i]];
            int              k  = std::min(B - 1, int((it.c[axis] - cb.lo[axis]) * scale));
            bins[k].grow(it.b);
            cnt[k]++;
        }
        float    rightArea[B];
        uint32_t rightCnt[B];
        Box      acc;
        uint32_t ac = 0;
        for (int k = B - 1; k > 0; --k)
        {
            acc.grow(bins[k]);
            ac += cnt[k];
            rightArea[k] = acc.area();
            rightCnt[k]  = ac;
        }
        Box      lacc;
        uint32_t lc = 0;
        for (int k = 0; k < B - 1; ++k)
        {
            lacc.grow(bins[k]);
            lc += cnt[k];
            if (lc == 0 || rightCnt[k + 1] == 0) continue;
            float cost = lacc.area() * float(lc) + rightArea[k + 1] * float(rightCnt[k + 1]);
            if (cost < best)
            {
                best      = cost;
                bestAxis  = axis;
                bestSplit = k;
            }
        }
    }
    uint32_t mid;
    if (bestAxis < 0)
    {
        // All centroids coincide: split in the middle of the list.
        mid = begin + n / 2;
    }
    else
    {
        float ext   = cb.hi[bestAxis] - cb.lo[bestAxis];
        float scale = float(B) / ext;
        auto  pivot = std::partition(ids.begin() + begin, ids.begin() + end, [&](uint32_t id) {
            int k = std::min(B - 1, int((items[id].c[bestAxis] - cb.lo[bestAxis]) * scale));
            return k <= bestSplit;
        });
        mid = uint32_t(pivot - ids.begin());
        if (mid == begin || mid == end) mid = begin + n / 2;
    }
    uint32_t l  = nodeCount.fetch_add(2);
    node.left   = l;
    node.count  = 0;
    bool spawn  = n > 200000;
    if (spawn)
    {
        std::thread th([&, l, begin, mid, depth]() { buildRec(s, items, ids, begin, mid, l, nodeCount, depth + 1); });
        buildRec(s, items, ids, mid, end, l + 1, nodeCount, depth + 1);
        th.join();
    }
    else
    {
        buildRec(s, items, ids, begin, mid, l, nodeCount, depth + 1);
        buildRec(s, items, ids, mid, end, l + 1, nodeCount, depth + 1);
    }
}

void buildBVH(Scene& s)
{
    uint32_t               n = s.ntris;
    std::vector<BuildItem> items(n);
    for (uint32_t i = 0; i < n; ++i)
    {
        const float* t = &s.tri[9 * size_t(i)];
        Box          b;
        b.grow(t);
        b.grow(t + 3);
        b.grow(t + 6);
        for (int a = 0; a < 3; ++a)
        {
            float m = std::max(std::abs(b.lo[a]), std::abs(b.hi[a]));
            float e = m * 9.5367431640625e-07f + 1e-30f; // 2^-20 relative
            b.lo[a] -= e;
            b.hi[a] += e;
            items[i].c[a] = 0.5f * (b.lo[a] + b.hi[a]);
        }
        items[i].b = b;
    }
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; ++i) ids[i] = i;
    s.nodes.assign(std::max<size_t>(1, 2 * size_t(n)), Node{});
    std::atomic<uint32_t> count{1};
    if (n > 0) buildRec(s, items, ids, 0, n, 0, count, 0);
    s.nodes.resize(count.load());
    s.order = ids;
}

struct RayQ
{
    RayPre pre;
    float  inv[3];
    float  tmin;
};

inline RayQ makeRay(V3<float> o, V3<float> d, float tmin)
{
    RayQ r;
    r.pre  = rayPrepare(o, d);
    r.tmin = tmin;
    for (int a = 0; a < 3; ++a)
    {
        float da = d[a];
        if (std::abs(da) < 1e-30f) da = da < 0.0f ? -1e-30f : 1e-30f;
        r.inv[a] = 1.0f / da;
    }
    return r;
}

inline bool boxHit(const Box& b, const RayQ& r, float tmax, float* tnear)
{
    float t0 = -FLT_MAX, t1 = FLT_MAX;
    for (int a = 0; a < 3; ++a)
    {
        float ta = (b.lo[a] - r.pre.o[a]) * r.inv[a];
        float tb = (b.hi[a] - r.pre.o[a]) * r.inv[a];
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
    }
    t0 = t0 - std::abs(t0) * 1e-6f;
    t1 = t1 + std::abs(t1) * 1e-6f;
    *tnear = t0;
    return t0 <= t1 && t1 >= r.tmin && t0 <= tmax;
}

struct Hit
{
    float    t  = FLT_MAX;
    uint32_t id = 0xffffffffu;
    float    b1 = 0, b2 = 0;
};

// Closest hit in (tmin, tmax); equal t resolved to the lower triangle id.
inline void testTri(const Scene& s, const RayQ& r, uint32_t id, Hit& h)
{
    const float* t = &s.tri[9 * size_t(id)];
    float        tt, b1, b2;
    if (!intersectTri(r.pre, {t[0], t[1], t[2]}, {t[3], t[4], t[5]}, {t[6], t[7], t[8]}, &tt, &b1, &b2)) return;
    if (!(tt > r.tmin)) return;
    if (tt < h.t || (tt == h.t && id < h.id))
    {
        h.t  = tt;
        h.id = id;
        h.b1 = b1;
        h.b2 = b2;
    }
}

Hit closest(const Scene& s, V3<float> o, V3<float> d, float tmin, float tmax)
{
    Hit  h;
    h.t    = tmax;
    RayQ r = makeRay(o, d, tmin);
    if (s.ntris == 0) return h;
    uint32_t stack[128];
    int      sp = 0;
    stack[sp++] = 0;
    while (sp > 0)
    {
        const Node& n = s.nodes[stack[--sp]];
        float       tn;
        if (!boxHit(n.box, r, h.t, &tn)) continue;
        if (n.count)
        {
            for (uint32_t i = 0; i < n.count; ++i) testTri(s, r, s.order[n.first + i], h);
            continue;
        }
        float tl, tr;
        bool  hl = boxHit(s.nodes[n.left].box, r, h.t, &tl);
        bool  hr = boxHit(s.nodes[n.left + 1].box, r, h.t, &tr);
        if (hl && hr)
        {
            if (tl <= tr)
            {
                stack[sp++] = n.left + 1;
                stack[sp++] = n.left;
            }
            else
            {
                stack[sp++] = n.left;
                stack[sp++] = n.left + 1;
            }
        }
        else if (hl)
            stack[sp++] = n.left;
        else if (hr)
            stack[sp++] = n.left + 1;
    }
    return h;
}

bool occluded(const Scene& s, V3<float> o, V3<float> d, float tmin, float tmax)
{
    if (s.ntris == 0) return false;
    RayQ     r = makeRay(o, d, tmin);
    uint32_t stack[128];
    int      sp = 0;
    stack[sp++] = 0;
    while (sp > 0)
    {
        const Node& n = s.nodes[stack[--sp]];
        float       tn;
        if (!boxHit(n.box, r, tmax, &tn)) continue;
        if (n.count)
        {
            for (uint32_t i = 0; i < n.count; ++i)
            {
                const float* t = &s.tri[9 * size_t(s.order[n.first + i])];
                float        tt, b1, b2;
                if (intersectTri(r.pre, {t[0], t[1], t[2]}, {t[3], t[4], t[5]}, {t[6], t[7], t[8]}, &tt, &b1, &b2) &&
                    tt > tmin && tt < tmax)
                    return true;
            }
            continue;
        }
        stack[sp++] = n.left;
        stack[sp++] = n.left + 1;
    }
    return false;
}

Hit bruteforce(const Scene& s, V3<float> o, V3<float> d, float tmin, float tmax)
{
    Hit h;
    h.t    = tmax;
    RayQ r = makeRay(o, d, tmin);
    for (uint32_t i = 0; i < s.ntris; ++i) testTri(s, r, i, h);
    return h;
}

} // namespace

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
extern "C" {

// Layouts shared with the product's C ABI (include/colvillea_b200.h):
//   material: 16 floats {type, r, g, b, roughness, etaInt, eta.xyz, k.xyz,
//             reflectance, roughness and normal-map texture (1-based, 0 none), 0};
//             alpha = roughness^2 (metal.h:52, glass.h:26).
//   texture : orc_texture {format 0 RGBA8 / 1 RGBA32F, w, h, srgb, texels}.
//   emitter : 12 floats {type(0 dir, 1 dome), intensity.xyz, direction.xyz,
//             angularRadius, domeW, domeH, 0, 0}; dome texels separate.
struct orc_scene_desc
{
    const float*    pos;
    const float*    nrm;
    const float*    tan;
    const float*    uv;
    uint32_t        nverts;
    const uint32_t* idx;
    const uint32_t* tri_material;
    uint32_t        ntris;
    const float*    materials;
    uint32_t        nmaterials;
    const float*    emitters;
    uint32_t        nemitters;
    const float*    dome_texels; // RGBA32F
    const float*    camera;      // pos, d00, ddu, ddv (12 floats)
    const orc::Texture* textures;
    uint32_t        ntextures;
};

// Integrator flags.
enum
{
    ORC_COMPAT_PDF       = 1u << 0, // the reference's pdf functions (conductor pdfAll(wo), diffuse cos(wo), dielectric extra cos(H))
    ORC_COMPAT_FRAME     = 1u << 1, // PT only: shading-frame normal = geometric normal (the reference's swapped arguments)
    ORC_COMPAT_ESCAPE    = 1u << 2, // Q5 + Q6 + Q9 + Q12 (reference MIS/escape bookkeeping)
    ORC_DOME_ALIAS       = 1u << 4, // the GPU's alias-table dome sampler (tables set by orc_scene_set_dome_tables)
    ORC_DIRECT_LIGHTING  = 1u << 8,
};

struct orc_config
{
    uint32_t max_depth;      // ray segments per path (path.cpp:135: 5)
    uint32_t rr_start_depth; // 0 = no Russian roulette
    uint32_t flags;
    uint32_t frame0;
};

void* orc_scene_create(const orc_scene_desc* d)
{
    auto s     = new Scene();
    s->ntris   = d->ntris;
    s->mesh    = MeshView{d->pos, d->nrm, d->tan, d->uv, d->idx};
    s->triMaterial = d->tri_material;
    s->tri.resize(9 * size_t(d->ntris));
    for (uint32_t i = 0; i < d->ntris; ++i)
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a) s->tri[9 * size_t(i) + 3 * v + a] = d->pos[3 * size_t(d->idx[3 * size_t(i) + v]) + a];
    buildBVH(*s);
    for (uint32_t m = 0; m < d->nmaterials; ++m)
    {
        const float* p = d->materials + 16 * size_t(m);
        Bsdf<float>  b{};
        b.type   = uint32_t(p[0]);
        b.r      = {p[1], p[2], p[3]};
        float rg = p[4];
        b.alpha  = rg * rg;
        b.etaInt = p[5];
        b.eta    = {p[6], p[7], p[8]};
        b.k      = {p[9], p[10], p[11]};
        b.etaExt = 1.0f;
        s->materials.push_back(b);
        s->matTex.push_back({uint32_t(p[12]), uint32_t(p[13]), uint32_t(p[14])});
    }
    s->textures.assign(d->textures, d->textures + d->ntextures);
    for (uint32_t e = 0; e < d->nemitters; ++e)
    {
        const float* p = d->emitters + 12 * size_t(e);
        Scene::Em    em{};
        em.type = int(p[0]);
        if (em.type == 0)
            em.dir = Directional{{p[1], p[2], p[3]}, {p[4], p[5], p[6]}, p[7]};
        else
        {
            int w = int(p[8]), h = int(p[9]);
            s->domeTex.assign(d->dome_texels, d->dome_texels + 4 * size_t(w) * h);
            buildDomeTables(s->domeTex.data(), w, h, s->pU, s->cU, s->pV, s->cV);
            s->dome    = Dome{w, h, s->domeTex.data(), s->pU.data(), s->cU.data(), s->pV.data(), s->cV.data()};
            s->hasDome = true;
        }
        s->emitters.push_back(em);
    }
    const float* c = d->camera;
    s->camPos      = {c[0], c[1], c[2]};
    s->d00         = {c[3], c[4], c[5]};
    s->ddu         = {c[6], c[7], c[8]};
    s->ddv         = {c[9], c[10], c[11]};
    return s;
}

void orc_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

uint32_t orc_scene_bvh_nodes(void* s) { return uint32_t(static_cast<Scene*>(s)->nodes.size()); }

// Dome tables as built by the reference's FP32 preprocessing.
void orc_scene_dome_tables(void* sp, float* pU, float* cU, float* pV, float* cV)
{
    Scene* s = static_cast<Scene*>(sp);
    std::copy(s->pU.begin(), s->pU.end(), pU);
    std::copy(s->cU.begin(), s->cU.end(), cU);
    std::copy(s->pV.begin(), s->pV.end(), pV);
    std::copy(s->cV.begin(), s->cV.end(), cV);
}

// Replaces the scene's dome tables with given ones (e.g. the GPU build's
// FP64-built tables, rounded to FP32) and adds the alias tables used under
// ORC_DOME_ALIAS; sizes as orc_scene_dome_tables, alias tables 2 uint32 per
// entry (h per row, w*h per column).  Returns 0, or -1 without a dome.
int orc_scene_set_dome_tables(void* sp, const float* pU, const float* cU, const float* pV, const float* cV,
                              const uint32_t* aliasRow, const uint32_t* aliasCol)
{
    Scene* s = static_cast<Scene*>(sp);
    if (!s->hasDome) return -1;
    const size_t w = size_t(s->dome.w), h = size_t(s->dome.h);
    s->pU.assign(pU, pU + (w + 1) * h);
    s->cU.assign(cU, cU + (w + 1) * h);
    s->pV.assign(pV, pV + h + 1);
    s->cV.assign(cV, cV + h + 1);
    if (aliasRow && aliasCol)
    {
        s->aliasRow.assign(aliasRow, aliasRow + 2 * h);
        s->aliasCol.assign(aliasCol, aliasCol + 2 * w * h);
    }
    s->dome.pUcondV_c = s->pU.data();
    s->dome.cdfU      = s->cU.data();
    s->dome.pV_c      = s->pV.data();
    s->dome.cdfV      = s->cV.data();
    s->dome.aliasRow  = s->aliasRow.empty() ? nullptr : s->aliasRow.data();
    s->dome.aliasCol  = s->aliasCol.empty() ? nullptr : s->aliasCol.data();
    return 0;
}

// rays: 8 floats each {o.xyz, tmin, d.xyz, tmax}.
void orc_trace(void* sp, const float* rays, uint32_t n, int bruteforce, float* t, uint32_t* id, float* b1, float* b2,
               int threads)
{
    Scene* s = static_cast<Scene*>(sp);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < int64_t(n); ++i)
    {
        const float* r = rays + 8 * i;
        Hit h = bruteforce ? ::bruteforce(*s, {r[0], r[1], r[2]}, {r[4], r[5], r[6]}, r[3], r[7])
                           : closest(*s, {r[0], r[1], r[2]}, {r[4], r[5], r[6]}, r[3], r[7]);
        t[i]  = h.t;
        id[i] = h.id;
        b1[i] = h.b1;
        b2[i] = h.b2;
    }
}

void orc_occluded(void* sp, const float* rays, uint32_t n, uint8_t* occ, int threads)
{
    Scene* s = static_cast<Scene*>(sp);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < int64_t(n); ++i)
    {
        const float* r = rays + 8 * i;
        occ[i]         = occluded(*s, {r[0], r[1], r[2]}, {r[4], r[5], r[6]}, r[3], r[7]) ? 1 : 0;
    }
}

} // extern "C"

namespace
{
struct Counters
{
    uint64_t closest = 0, shadow = 0;
};

inline V3<float> emitterSample(const Scene& s, const Scene::Em& e, V2<float> u, V3<float>* dir, float* pdf, bool alias)
{
    if (e.type == 0) return directionalSample(e.dir, u, dir, pdf);
    return domeSample(s.dome, u, dir, pdf, alias);
}

inline float maxComp(V3<float> v)
{
    float m = v.x;
    if (v.y > m) m = v.y;
    if (v.z > m) m = v.z;
    return m;
}

// One camera path (PT) or one camera sample (DL); returns its radiance.
V3<float> tracePath(const Scene& s, const orc_config& cfg, uint32_t W, uint32_t H, uint32_t px, uint32_t py,
                    uint32_t frame, Counters& cnt)
{
    const bool compatPdf    = cfg.flags & ORC_COMPAT_PDF;
    const bool compatFrame  = cfg.flags & ORC_COMPAT_FRAME;
    const bool compatEscape = cfg.flags & ORC_COMPAT_ESCAPE;
    const bool dl           = cfg.flags & ORC_DIRECT_LIGHTING;
    const bool alias        = (cfg.flags & ORC_DOME_ALIAS) && !s.aliasRow.empty();
    const uint32_t N        = uint32_t(s.emitters.size());

    Rng       rng{px, py, frame, 0};
    V2<float> j = rng.next2D();
    V2<float> screen{(float(px) + j.x) / float(W), (float(py) + j.y) / float(H)};
    V3<float> d = s.d00 + screen.x * s.ddu;
    d           = d + screen.y * s.ddv;
    d           = normalize(d);
    V3<float> o = s.camPos;
    float     tmin = 0.0f;

    V3<float> L{0, 0, 0}, T{1, 1, 1}, E{0, 0, 0};
    for (uint32_t depth = 1;; ++depth)
    {
        cnt.closest++;
        Hit h = closest(s, o, d, tmin, FLT_MAX);
        if (h.id == 0xffffffffu)
        {
            // evaluateEscapedRays (raygeneration.cu:105-136)
            if (s.hasDome)
            {
                V3<float> Le = domeEval(s.dome, d, !compatEscape);
                if (depth == 1)
                    L = L + Le;
                else if (compatEscape)
                    L = L + T * (Le * E);
                else
                {
                    float pd = domePdf(s.dome, d, true) / float(N);
                    float w  = E.x / (E.x + pd);
                    L        = L + T * (Le * w);
                }
            }
            break;
        }
        if (!dl && depth == cfg.max_depth) break;

        HitAttr     a    = hitAttributes(s.mesh, h.id, h.b1, h.b2);
        uint32_t    mi   = s.triMaterial[h.id];
        Bsdf<float> bsdf = s.materials[mi];
        const auto& tx   = s.matTex[mi];
        // Material::getBSDF(uv): textures replace the constants (diffusemtl.h:22-27, metal.h:40-52).
        if (tx[0])
        {
            F4 c   = texUnit(s.textures[tx[0] - 1], a.uv.x, a.uv.y);
            bsdf.r = {c.v[0], c.v[1], c.v[2]};
        }
        if (tx[1])
        {
            float r    = texUnit(s.textures[tx[1] - 1], a.uv.x, a.uv.y).v[0];
            bsdf.alpha = r * r;
        }
        V3<float>    wo = -d;
        V2<float>    u  = rng.next2D();
        // Material::getShadingFrame (material.h:128-147) with the path-tracing
        // call site's swapped (ng, ns) (raygeneration.cu:324-330): without a
        // normal map the compat frame's normal is ng; a normal map's tangent
        // frame and pull-up use ns.  The direct-lighting kernel ignores normal
        // maps (raygeneration.cu:179,237).
        Frame<float> fr;
        if (tx[2] && !(dl && compatFrame))
        {
            F4 nt = texUnit(s.textures[tx[2] - 1], a.uv.x, a.uv.y);
            fr    = normalMappedFrame(wo, a.dpdu, a.dpdv, a.ns, V3<float>{nt.v[0], nt.v[1], nt.v[2]}, bsdf.type != 2u);
        }
        else
            fr = Frame<float>{a.dpdv, a.dpdu, (!dl && compatFrame) ? a.ng : a.ns};

        // Emitter sampling with MIS (raygeneration.cu:332-384 / 174-227).
        if (N > 0)
        {
            uint32_t  pick = uint32_t(std::floor(u.x * float(N)));
            V2<float> us{u.x * float(N) - float(pick), u.y};
            V3<float> ldir{0, 0, 0};
            float     lpdf  = 0.0f;
            const auto& em  = s.emitters[pick];
            V3<float> value = emitterSample(s, em, us, &ldir, &lpdf, alias);
            if (compatEscape) value = value * float(N);
            if (lpdf == 0.0f) value = {0, 0, 0};
            if (nonzero(value) && lpdf > 0.0f)
            {
                V3<float> wiL = fr.toLocal(ldir), woL = fr.toLocal(wo);
                V3<float> f   = bsdfEval(bsdf, woL, wiL);
                if (nonzero(f))
                {
                    float bp = bsdfPdf(bsdf, woL, wiL, compatPdf);
                    float c  = dl && compatEscape ? cosTheta(wiL) : std::abs(cosTheta(wiL));
                    V3<float> Li;
                    if (compatEscape)
                    {
                        float w = misBalanced(lpdf, bp);
                        V3<float> base = dl ? value : T * value;
                        Li = base * f;
                        Li = Li * c;
                        Li = Li * w;
                        Li = Li / lpdf;
                    }
                    else
                    {
                        float pl = lpdf / float(N);
                        float w  = em.type == 1 ? misBalanced(pl, bp) : 1.0f;
                        V3<float> base = dl ? value : T * value;
                        Li = base * f;
                        Li = Li * c;
                        Li = Li * w;
                        Li = Li / pl;
                    }
                    cnt.shadow++;
                    if (!occluded(s, a.p, ldir, 0.001f, FLT_MAX)) L = L + Li;
                }
            }
        }

        // BSDF sampling with MIS (raygeneration.cu:391-455 / 234-281).
        V2<float> u2  = rng.next2D();
        V3<float> woL = fr.toLocal(wo);
        V3<float> wiL{0, 0, 0};
        float     bp = 0.0f;
        V3<float> f  = bsdfSample(bsdf, woL, u2, &wiL, &bp);
        // The corrected estimator stops paths whose sampled pdf is not
        // positive; the reference divides by it (raygeneration.cu:430).
        if (!nonzero(f) || (!compatEscape && !(bp > 0.0f))) break;
        V3<float> dir = fr.toWorld(wiL);
        float     lightPdf = s.hasDome ? domePdf(s.dome, dir, !compatEscape) : 0.0f;
        if (dl)
        {
            // Second shadow queue: BSDF-sampled dome light (raygeneration.cu:245-281).
            if (!s.hasDome) break;
            float c = compatEscape ? cosTheta(wiL) : std::abs(cosTheta(wiL));
            float pl = compatEscape ? lightPdf : lightPdf / float(N);
            if (compatEscape && !(lightPdf > 0.0f)) break;
            V3<float> Ld = domeEval(s.dome, dir, !compatEscape);
            float     w  = misBalanced(bp, pl);
            float     k0 = f.x * c, k1 = f.y * c, k2 = f.z * c;
            V3<float> kk{k0 * w / bp, k1 * w / bp, k2 * w / bp};
            Ld = Ld * kk;
            cnt.shadow++;
            if (!occluded(s, a.p, dir, 0.001f, FLT_MAX)) L = L + Ld;
            break;
        }
        float c = std::abs(cosTheta(wiL));
        V3<float> tk{f.x * c / bp, f.y * c / bp, f.z * c / bp};
        T = T * tk;
        if (cfg.rr_start_depth > 0 && depth >= cfg.rr_start_depth)
        {
            float q = maxComp(T);
            q       = q < 1.0f ? q : 1.0f;
            float r = rng.next1D();
            if (r >= q) break;
            T = T / q;
        }
        if (compatEscape)
        {
            if (!(lightPdf > 0.0f)) break; // the reference continues a path only where the dome pdf is non-zero
            float w = misBalanced(bp, lightPdf);
            E       = {f.x * c * w / bp, f.y * c * w / bp, f.z * c * w / bp};
        }
        else
            E = {bp, 0.0f, 0.0f};
        o    = a.p;
        d    = dir;
        tmin = 0.001f; // kRayTOffsetEpsilon, config.h:11
    }
    return L;
}

} // namespace

extern "C" {

// Renders `spp` samples per pixel (frames frame0 .. frame0+spp-1) for the
// listed pixels (all pixels when `pixels` is null), accumulating per-pixel
// FP64 sum and sum of squares of the per-sample radiance (3 channels each).
// counters (optional): {closest rays, shadow rays}.
void orc_render(void* sp, const orc_config* cfg, uint32_t W, uint32_t H, uint32_t spp, const uint32_t* pixels,
                uint32_t npix, double* sum, double* sumsq, int threads, uint64_t* counters)
{
    const Scene& s     = *static_cast<Scene*>(sp);
    uint32_t     n     = pixels ? npix : W * H;
    uint64_t     total = 0, shadow = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : total, shadow)
    {
        Counters cnt;
#pragma omp for schedule(dynamic, 16)
        for (int64_t i = 0; i < int64_t(n); ++i)
        {
            uint32_t pix = pixels ? pixels[i] : uint32_t(i);
            uint32_t px = pix % W, py = pix / W;
            double   s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
            for (uint32_t k = 0; k < spp; ++k)
            {
                V3<float> L = tracePath(s, *cfg, W, H, px, py, cfg->frame0 + k, cnt);
                for (int c = 0; c < 3; ++c)
                {
                    s1[c] += double(L[c]);
                    s2[c] += double(L[c]) * double(L[c]);
                }
            }
            for (int c = 0; c < 3; ++c)
            {
                sum[3 * size_t(i) + c]   = s1[c];
                sumsq[3 * size_t(i) + c] = s2[c];
            }
        }
        total += cnt.closest;
        shadow += cnt.shadow;
    }
    if (counters)
    {
        counters[0] = total;
        counters[1] = shadow;
    }
}

// --- unit functions (batch), float path; see orc_core.h / orc_emit.h -------
// BSDF params: 11 floats {r.xyz, alpha, etaInt, eta.xyz, k.xyz}.
static Bsdf<float> bsdfFrom(int type, const float* p)
{
    Bsdf<float> b{};
    b.type   = uint32_t(type);
    b.r      = {p[0], p[1], p[2]};
    b.alpha  = p[3];
    b.etaInt = p[4];
    b.eta    = {p[5], p[6], p[7]};
    b.k      = {p[8], p[9], p[10]};
    b.etaExt = 1.0f;
    return b;
}
static Bsdf<double> bsdfFromD(int type, const float* p)
{
    Bsdf<double> b{};
    b.type   = uint32_t(type);
    b.r      = {p[0], p[1], p[2]};
    b.alpha  = p[3];
    b.etaInt = p[4];
    b.eta    = {p[5], p[6], p[7]};
    b.k      = {p[8], p[9], p[10]};
    b.etaExt = 1.0;
    return b;
}

void orc_bsdf_eval(int type, const float* params, const float* wo, const float* wi, float* out, int n, int fp64,
                   double* out64)
{
    for (int i = 0; i < n; ++i)
    {
        if (fp64)
        {
            V3<double> r = bsdfEval(bsdfFromD(type, params + 11 * i), V3<double>{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]},
                                    V3<double>{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]});
            for (int c = 0; c < 3; ++c) out64[3 * i + c] = r[c];
        }
        else
        {
            V3<float> r = bsdfEval(bsdfFrom(type, params + 11 * i), ld3(wo, i), ld3(wi, i));
            for (int c = 0; c < 3; ++c) out[3 * i + c] = r[c];
        }
    }
}

void orc_bsdf_pdf(int type, const float* params, const float* wo, const float* wi, float* out, int n, int compat,
                  int fp64, double* out64)
{
    for (int i = 0; i < n; ++i)
    {
        if (fp64)
            out64[i] = bsdfPdf(bsdfFromD(type, params + 11 * i), V3<double>{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]},
                               V3<double>{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]}, compat != 0);
        else
            out[i] = bsdfPdf(bsdfFrom(type, params + 11 * i), ld3(wo, i), ld3(wi, i), compat != 0);
    }
}

void orc_bsdf_sample(int type, const float* params, const float* wo, const float* u2, float* wi_out, float* pdf_out,
                     float* val_out, int n, int fp64, double* wi64, double* pdf64, double* val64)
{
    for (int i = 0; i < n; ++i)
    {
        if (fp64)
        {
            V3<double> wi{0, 0, 0};
            double     pdf = 0;
            V3<double> v   = bsdfSample(bsdfFromD(type, params + 11 * i), V3<double>{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]},
                                        V2<double>{u2[2 * i], u2[2 * i + 1]}, &wi, &pdf);
            for (int c = 0; c < 3; ++c)
            {
                wi64[3 * i + c]  = wi[c];
                val64[3 * i + c] = v[c];
            }
            pdf64[i] = pdf;
        }
        else
        {
            V3<float> wi{0, 0, 0};
            float     pdf = 0;
            V3<float> v   = bsdfSample(bsdfFrom(type, params + 11 * i), ld3(wo, i), V2<float>{u2[2 * i], u2[2 * i + 1]}, &wi, &pdf);
            for (int c = 0; c < 3; ++c)
            {
                wi_out[3 * i + c]  = wi[c];
                val_out[3 * i + c] = v[c];
            }
            pdf_out[i] = pdf;
        }
    }
}

void orc_ggx_eval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1wi, float* G,
                  float* pdfAll, int n)
{
    for (int i = 0; i < n; ++i)
    {
        GGX<float> d(alpha[i]);
        V3<float>  mm = ld3(m, i), a = ld3(wi, i), b = ld3(wo, i);
        D[i]      = d.D(mm);
        G1wi[i]   = d.smithG1(a, mm);
        G[i]      = d.G(a, b, mm);
        pdfAll[i] = d.pdfAll(mm);
    }
}

void orc_ggx_sample(const float* alpha, const float* u2, float* m_out, float* pdf_out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        GGX<float> d(alpha[i]);
        float      pdf = 0;
        V3<float>  m   = d.sampleAll(V2<float>{u2[2 * i], u2[2 * i + 1]}, &pdf);
        for (int c = 0; c < 3; ++c) m_out[3 * i + c] = m[c];
        pdf_out[i] = pdf;
    }
}

void orc_fresnel_conductor(const float* cosi, const float* eta, const float* k, float* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        V3<float> r = fresnelConductor(cosi[i], ld3(eta, i), ld3(k, i));
        for (int c = 0; c < 3; ++c) out[3 * i + c] = r[c];
    }
}

void orc_fresnel_dielectric(const float* cosi, const float* eta, float* F, float* cost, int n)
{
    for (int i = 0; i < n; ++i)
    {
        float ct = 0;
        F[i]     = fresnelDielectricExt(cosi[i], &ct, eta[i]);
        cost[i]  = ct;
    }
}

void orc_warp(const float* u2, float* disk2, float* hemi3, int n)
{
    for (int i = 0; i < n; ++i)
    {
        V2<float> s{u2[2 * i], u2[2 * i + 1]};
        V2<float> d      = concentricDisk(s);
        disk2[2 * i]     = d.x;
        disk2[2 * i + 1] = d.y;
        V3<float> h      = cosineHemisphere(s);
        for (int c = 0; c < 3; ++c) hemi3[3 * i + c] = h[c];
    }
}

void orc_make_frame(const float* a, float* b, float* c, int n)
{
    for (int i = 0; i < n; ++i)
    {
        V3<float> bb, cc;
        makeFrame(ld3(a, i), &bb, &cc);
        for (int k = 0; k < 3; ++k)
        {
            b[3 * i + k] = bb[k];
            c[3 * i + k] = cc[k];
        }
    }
}

void orc_frame(const float* s, const float* t, const float* nrm, const float* v, float* local, float* world, int n)
{
    for (int i = 0; i < n; ++i)
    {
        Frame<float> f{ld3(s, i), ld3(t, i), ld3(nrm, i)};
        V3<float>    l = f.toLocal(ld3(v, i)), w = f.toWorld(ld3(v, i));
        for (int k = 0; k < 3; ++k)
        {
            local[3 * i + k] = l[k];
            world[3 * i + k] = w[k];
        }
    }
}

void orc_pcg4d(const uint32_t* in, uint32_t* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        uint32_t v[4] = {in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]};
        pcg4d(v);
        for (int k = 0; k < 4; ++k) out[4 * i + k] = v[k];
    }
}

void orc_sampler_sequence(const uint32_t* pxpyframe, int n, int m, float* out)
{
    for (int i = 0; i < n; ++i)
    {
        Rng r{pxpyframe[3 * i], pxpyframe[3 * i + 1], pxpyframe[3 * i + 2], 0};
        for (int j = 0; j < m; ++j) out[size_t(i) * m + j] = r.next1D();
    }
}

// Dome functions against caller-supplied tables (same layout as the reference).
void orc_dome_build_tables(const float* texels, int w, int h, float* pU, float* cU, float* pV, float* cV)
{
    std::vector<float> a, b, c, d;
    buildDomeTables(texels, w, h, a, b, c, d);
    std::copy(a.begin(), a.end(), pU);
    std::copy(b.begin(), b.end(), cU);
    std::copy(c.begin(), c.end(), pV);
    std::copy(d.begin(), d.end(), cV);
}

void orc_dome_sample(const float* texels, int w, int h, const float* pU, const float* cU, const float* pV,
                     const float* cV, const float* u2, float* dir, float* pdf, float* val, int n)
{
    Dome d{w, h, texels, pU, cU, pV, cV};
    for (int i = 0; i < n; ++i)
    {
        V3<float> dd{0, 0, 0};
        float     p = 0;
        V3<float> v = domeSample(d, V2<float>{u2[2 * i], u2[2 * i + 1]}, &dd, &p);
        for (int k = 0; k < 3; ++k)
        {
            dir[3 * i + k] = dd[k];
            val[3 * i + k] = v[k];
        }
        pdf[i] = p;
    }
}

void orc_dome_pdf_eval(const float* texels, int w, int h, const float* pU, const float* pV, const float* dirs, float* pdf,
                       float* val, int n)
{
    Dome d{w, h, texels, pU, nullptr, pV, nullptr};
    for (int i = 0; i < n; ++i)
    {
        V3<float> dd = ld3(dirs, i);
        pdf[i]       = domePdf(d, dd);
        V3<float> v  = domeEval(d, dd);
        for (int k = 0; k < 3; ++k) val[3 * i + k] = v[k];
    }
}

void orc_directional_sample(const float* params /*7: intensity, direction, radius*/, const float* u2, float* dir,
                            float* pdf, float* val, int n)
{
    Directional e{{params[0], params[1], params[2]}, {params[3], params[4], params[5]}, params[6]};
    for (int i = 0; i < n; ++i)
    {
        V3<float> dd{0, 0, 0};
        float     p = 0;
        V3<float> v = directionalSample(e, V2<float>{u2[2 * i], u2[2 * i + 1]}, &dd, &p);
        for (int k = 0; k < 3; ++k)
        {
            dir[3 * i + k] = dd[k];
            val[3 * i + k] = v[k];
        }
        pdf[i] = p;
    }
}

void orc_texture_lookup(const orc::Texture* t, const float* uv, float* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        F4 c = texUnit(*t, uv[2 * i], uv[2 * i + 1]);
        for (int k = 0; k < 4; ++k) out[4 * i + k] = c.v[k];
    }
}

// in: 16 floats per item {wo, dpdu, dpdv, nb, texel rgb, pullUp}; out 9 {s, t, n}.
void orc_normal_frame(const float* in, float* out, int n, int fp64)
{
    for (int i = 0; i < n; ++i)
    {
        const float* p = in + 16 * size_t(i);
        float*       o = out + 9 * size_t(i);
        if (fp64)
        {
            auto v = [&](int k) { return V3<double>{p[k], p[k + 1], p[k + 2]}; };
            Frame<double> f = normalMappedFrame(v(0), v(3), v(6), v(9), v(12), p[15] != 0.0f);
            V3<double> r[3] = {f.s, f.t, f.n};
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) o[3 * k + c] = float(r[k][c]);
        }
        else
        {
            auto v = [&](int k) { return V3<float>{p[k], p[k + 1], p[k + 2]}; };
            Frame<float> f = normalMappedFrame(v(0), v(3), v(6), v(9), v(12), p[15] != 0.0f);
            V3<float> r[3] = {f.s, f.t, f.n};
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) o[3 * k + c] = r[k][c];
        }
    }
}

void orc_hit_attributes(const float* pos, const float* nrm, const float* tan, const float* uv, const uint32_t* idx,
                        const uint32_t* prim, const float* b1, const float* b2, float* out /*17 per hit*/, int n)
{
    MeshView m{pos, nrm, tan, uv, idx};
    for (int i = 0; i < n; ++i)
    {
        HitAttr a = hitAttributes(m, prim[i], b1[i], b2[i]);
        float*  o = out + 17 * size_t(i);
        V3<float> v[5] = {a.p, a.ng, a.ns, a.dpdu, a.dpdv};
        for (int k = 0; k < 5; ++k)
            for (int c = 0; c < 3; ++c) o[3 * k + c] = v[k][c];
        o[15] = a.uv.x;
        o[16] = a.uv.y;
    }
}

} // extern "C"
