// The wavefront integrator (host side) and its device-visible layouts.
#pragma once

#include "cl_bvh.cuh"
#include "cl_dome.h"
#include "cl_guide.h"
#include "cl_internal.h"
#include "cl_texture.h"

#include <memory>
#include <vector>

namespace clb
{
struct ClassifyView;
constexpr int      kMaxEmitters = 8;
constexpr uint32_t kLastFlag    = 0x80000000u; // shadow entry: path ends after this shadow query

struct EmitterDev
{
    uint32_t         type; // 0 directional, 1 dome
    DirectionalLight dl;
};

constexpr uint32_t kMatF4 = 4; // material record: {type, r.xyz} {alpha, etaInt, eta.xy} {eta.z, k.xyz} {textures}

struct SceneDev
{
    BvhView bvh;
    const uint4* __restrict__ triIdx;  // per primitive: i0, i1, i2, material
    const float4* __restrict__ vtx;    // 3 per vertex: {p.xyz, n.x} {n.y, n.z, t.x, t.y} {t.z, u, v, flags}
    const float4* __restrict__ mats;   // kMatF4 per material; the last holds the 1-based texture indices
                                       // {reflectance, roughness, normal map, 0} as uint bits
    const unsigned long long* __restrict__ tex; // cudaTextureObject_t per texture
    DomeView   dome;
    int        hasDome;
    uint32_t   numEmitters;
    EmitterDev emitters[kMaxEmitters];
};

// Per-render values, in device memory so that captured graphs stay valid.
struct WaveParams
{
    uint32_t           W, H, frame0, maxDepth, rrStart, flags, dl;
    uint32_t           recStride; // guiding: slots s with s % recStride == 0 record training data (0: off)
    uint32_t           cacheTrain; // radiance cache: 1 = training paths are traced and recorded this pass
    uint32_t           pad3;
    unsigned long long totalPaths;
    float              cam[12];
};

struct Counters
{
    uint32_t           rayCount[2];
    uint32_t           shadowCount;
    uint32_t           fetchTrace, fetchShadow; // traversal kernels' ray supplies
    uint32_t           error;
    uint32_t           classCount[4]; // per shading class: diffuse, conductor, dielectric, escaped
    unsigned long long pathNext;
    unsigned long long raysClosest, raysShadow;
    unsigned long long statNodes, statTris;
    unsigned long long statNodesS, statTrisS;
    uint32_t           fetchInfer; // guiding: inference fetch over the guided class queues
    uint32_t           recCount;   // guiding: training records appended (may exceed the capacity)
    uint32_t           trainCount; // guiding: records the training step reads (clamped)
    uint32_t           pad2;
    unsigned long long inferred;   // guiding: network evaluations
    uint32_t           cacheCount; // radiance cache: rays terminating into the cache this wave (compacted)
    uint32_t           cacheRec;   // radiance cache: training records appended (may exceed the capacity)
    uint32_t           cacheTrainCount; // radiance cache: records the training step reads (clamped)
    uint32_t           pad4;
    unsigned long long cacheQueries; // radiance cache: network evaluations
};

struct QueueDev
{
    float4*   rqO[2];
    float4*   rqD[2];
    uint32_t* rqSlot[2];
    float4*   hit;
    const uint4* hitIdx; // per ray: the hit triangle's {vertex ids, material} (written with the class queues)
    float4*   sqO;  // {o.xyz, slot | kLastFlag bits}
    float4*   sqD;  // {d.xyz, -}
    float4*   sqL;  // {Li.xyz, -}
    float4*   sqD2; // direct lighting: second (BSDF-sampled) shadow ray {d.xyz, valid}
    float4*   sqL2;
    uint32_t* classIdx; // 4 x slots ray-queue indices, sorted by shading class
    uint8_t*  vis;    // shadow ray visibility (1 = reaches the light), 2 per entry
    uint4*    psInfo; // {pixel, frame, depth | rngCounter << 8, -}
    float4*   psT;    // throughput
    float4*   psE;    // escape weight (compat) / BSDF pdf in .x
    float4*   psL;    // radiance so far
    float4*   film;
    double*   film64; // 6 per pixel: sum.rgb, sumsq.rgb
    Counters* ctr;
    uint32_t  slots;
    uint32_t  shadowCap;
};

// Guided path tracing: per-ray mixtures, per-slot vertex histories and the
// training records (no counterpart in the reference).
constexpr int kLobeF4 = 10; // 8 x {mu, kappa}, weights 0-3, weights 4-7
constexpr int kProbeF = 52; // floats per probed guide row
constexpr int kHistF4 = 5;  // {p, T.x} {n, T.y} {wo, T.z} {omega, BSDF pdf} {L snapshot, -}
struct GuideDev
{
    float4*  lobes;     // kLobeF4 per ray-queue index
    float4*  hist;      // (slots / recStride) x maxDepth x kHistF4
    float4*  rec;       // kRecordF4 per record
    uint32_t recCap;
    uint32_t classMask; // guided BSDF classes
    uint32_t minDepth;  // guided vertices have depth >= minDepth
    float    minAlpha;  // and, at conductors and dielectrics, GGX alpha >= minAlpha
    float*   probe;     // test probe (cl_integrator_guide_probe): per guided row k < probeCap,
    uint32_t probeCap;  // kProbeF floats {in9, ray index bits, 40 lobe floats, 2 pad}; null in renders
    float    boxScale;  // 1 / largest scene extent
    float    boxMin[3];
    uint32_t histDepth;
};

// Radiance cache (no counterpart in the reference): paths terminate into the
// cache at depth termDepth = prefix + 1; training paths (path index hash &
// trainMask == 0) continue to the maximum depth and record every vertex.
// psE.w of a slot holds kCacheTrainBit and the mask of recorded depths.
constexpr uint32_t kCacheTrainBit = 0x80000000u;
constexpr int      kCacheHistF4   = 4; // {p, T.x} {n, T.y} {wo, T.z} {L before the vertex's emitter sample, -}
struct CacheDev
{
    float4*   L;         // per ray-queue index: predicted outgoing radiance
    uint4*    enc;       // encoded inputs of the terminating rays (compacted)
    uint32_t* encIdx;    // their ray-queue indices
    float4*   hist;      // slots x histDepth x kCacheHistF4
    float4*   rec;       // kRecordF4 per training record
    uint32_t  recCap;
    uint32_t  termDepth; // 0: cache off
    uint32_t  trainMask;
    uint32_t  histDepth;
};

struct Params
{
    SceneDev          sc;
    QueueDev          q;
    GuideDev          g;
    CacheDev          c;
    const WaveParams* wp;
};

class Integrator
{
public:
    Integrator(cl_integrator_type type, uint32_t w, uint32_t h, const cl_render_config& cfg);
    ~Integrator();
    cl_status init(std::string* err);

    cl_status buildMeshes(const cl_mesh_desc* meshes, uint32_t n, std::string* err);
    cl_status buildInstances(const cl_instance_desc* inst, uint32_t n, std::string* err);
    cl_status updateMeshVertices(uint32_t meshId, const float* pos, const float* nrm, const float* tan, uint32_t count,
                                 uint32_t mode, std::string* err);
    cl_status buildMaterials(const cl_material_desc* m, uint32_t n, std::string* err);
    cl_status buildTextures(const cl_texture_desc* t, uint32_t n, std::string* err);
    cl_status buildEmitters(const cl_emitter_desc* e, uint32_t n, std::string* err);
    cl_status updateCamera(const cl_camera* c, std::string* err);
    cl_status render(uint32_t spp, std::string* err);
    cl_status readbackFilm(float* rgba, size_t bytes, std::string* err);
    cl_status readbackFilmAsync(float* rgba, size_t bytes, std::string* err);
    cl_status readbackWait(std::string* err);
    cl_status readbackFilmStats(double* sum, double* sumsq, size_t count, std::string* err);
    cl_status resize(uint32_t w, uint32_t h, std::string* err);
    cl_status resetIteration(std::string* err);
    cl_status setIteration(uint32_t iteration, std::string* err);
    void      stats(cl_stats* s) const;
    cl_status getBvh(void* nodes, size_t nodeBytes, void* tris, size_t triBytes, std::string* err);
    cl_status traceRays(const float* rays, uint32_t n, float* t, uint32_t* prim, float* b1, float* b2,
                        std::string* err);
    cl_status occludedRays(const float* rays, uint32_t n, uint8_t* occ, std::string* err);
    cl_status traceStats(const float* rays, uint32_t n, uint64_t* nodes, uint64_t* tris, std::string* err);
    cl_status domeTables(float* pU, float* cU, float* pV, float* cV, std::string* err);
    cl_status domeAliasTables(uint32_t* aliasRow, uint32_t* aliasCol, std::string* err);
    cl_status waveRays(uint64_t* out, uint32_t cap, uint32_t* count, std::string* err) const;
    cl_status guideProbe(uint32_t cap, float* rows, uint32_t* count, std::string* err);
    cl_status beginPass(uint32_t spp, bool record, bool cacheTrain, uint32_t* initSlots, std::string* err);
    cl_status domeAliasSample(const float* u2, float* dir, float* pdf, float* val, uint32_t n, std::string* err);

    cl_status setGuiding(const cl_guide_config* cfg, std::string* err);
    GuideNet* guideNet() const { return guide_.get(); }
    cl_status guideStats(cl_guide_stats* s, std::string* err) const;
    cl_status setRadianceCache(const cl_radiance_cache_config* cfg, std::string* err);
    CacheNet* cacheNet() const { return cache_.get(); }
    cl_status cacheStats(cl_guide_stats* s, std::string* err) const;

    uint32_t width() const { return W_; }
    uint32_t height() const { return H_; }

private:
    cl_status renderPass(uint32_t spp, bool record, bool cacheTrain, std::string* err);
    cl_status ensureGuideBuffers(std::string* err);
    cl_status ensureCacheBuffers(std::string* err);
    cl_status trainGuide(std::string* err);
    cl_status trainCache(std::string* err);
    cl_status ensureFilm(std::string* err);
    cl_status resolveFilm(std::string* err);
    cl_status ensureQueues(std::string* err);
    cl_status clearFilm(std::string* err);
    cl_status captureGraph(std::string* err);
    cl_status launchWave(int cur, bool profile, std::string* err);
    Params    params() const;
    ClassifyView classifyView() const;
    BvhView      bvhView() const;

    cl_integrator_type type_;
    uint32_t           W_, H_;
    cl_render_config   cfg_;
    cudaStream_t       stream_ = nullptr;
    int                numSMs_ = 148;
    int                traceBlocks_ = 0, shadeBlocks_ = 0, shadowBlocks_ = 0, traceBlocksTwo_ = 0;
    int                tBlocks() const { return twoLevel_ ? traceBlocksTwo_ : traceBlocks_; }

    // Meshes as given (host copies), flattened on instance build.
    struct HostMesh
    {
        std::vector<float>    pos, nrm, tan, uv;
        std::vector<uint32_t> idx;
        bool                  hasN = false, hasUV = false;
    };
    std::vector<HostMesh> meshes_;
    cl_status flattenInstance(const HostMesh& m, const float* M, uint32_t i, float* out, std::string* err);
    std::vector<cl_instance_desc> inst_;       // as built
    std::vector<uint32_t>         instVtxOff_; // first flattened vertex of each instance
    // Two-level scenes (CL_TWO_LEVEL): object-space pools, one tree per mesh,
    // the instance records; bvh_ is then the top tree over the instances.
    bool                   twoLevel_ = false;
    std::vector<std::unique_ptr<WideBvh>> blas_; // per mesh (null: not instanced)
    std::vector<uint32_t>  meshVtxBase_, meshTriBase_;
    DevBuf                 instDev_;
    uint32_t               twoLevelStack_ = 0;
    cl_status buildTwoLevel(const cl_instance_desc* inst, uint32_t n, std::string* err);
    cl_status uploadMeshPool(uint32_t meshId, std::string* err);
    cl_status buildBlas(uint32_t meshId, BuildArena* arena, cudaStream_t st, std::string* err);
    cl_status buildBlasAll(const std::vector<uint32_t>& meshes, std::string* err);
    cl_status buildTopLevel(BuildArena* arena, std::string* err);
    cl_status uploadInstances(std::string* err);
    cl_status updateTwoLevel(uint32_t meshId, uint32_t mode, std::string* err);
    void      instanceBox(uint32_t i, float* lo, float* hi) const;
    // Refit policy (CL_BVH_UPDATE_AUTO): rebuild when the refitted tree's
    // surface-area cost exceeds this multiple of the cost after its build.
    static constexpr double kRefitSahLimit = 1.5;
    double   sahBuild_ = 0.0, sah_ = 0.0;
    uint32_t refits_ = 0, rebuilds_ = 0;
    float    msBvhUpdate_ = 0.0f, msBvhRefit_ = 0.0f;

    // Device scene.
    DevBuf   triIdx_, vtx_, mats_, triPos_;
    WideBvh  bvh_;
    DomeTables dome_;
    bool     hasDome_ = false;
    std::vector<EmitterDev> emitters_;
    uint32_t numMaterials_ = 0;
    uint32_t numTris_      = 0;
    uint32_t maxMaterialIndex_ = 0;
    TextureSet textures_;
    uint32_t   maxTextureRef_ = 0; // largest 1-based texture index the materials use
    bool     sceneBuilt_   = false;

    // Film and wavefront state.
    DevBuf film_, film64_;
    // Film readback: mean radiance staged on the device, copied out on its own
    // stream so that a copy overlaps the next render.
    DevBuf       resolve_;
    cudaStream_t copyStream_ = nullptr;
    cudaEvent_t  evResolved_ = nullptr, evCopied_ = nullptr;
    DevBuf rqO_[2], rqD_[2], rqSlot_[2], hit_, hitIdx_, hitInst_, sqO_, sqD_, sqL_, sqD2_, sqL2_;
    DevBuf psInfo_, psT_, psE_, psL_, ctr_, wp_, vis_, classIdx_;
    uint32_t slots_ = 0, shadowCap_ = 0;
    WaveParams* hostWp_ = nullptr;   // pinned
    uint32_t*   hostCount_ = nullptr; // pinned
    cudaGraphExec_t graph_ = nullptr;
    bool            graphValid_ = false;

    cl_camera camera_{};
    bool      hasCamera_ = false;
    uint32_t  iteration_ = 0;
    uint32_t  filmSpp_   = 0;
    uint64_t  pathsDone_ = 0, raysClosest_ = 0, raysShadow_ = 0;
    uint32_t  waves_ = 0, launches_ = 0;
    uint64_t  lastNodes_ = 0, lastTris_ = 0, lastNodesS_ = 0, lastTrisS_ = 0, lastRaysC_ = 0, lastRaysS_ = 0;
    float     msBvh_ = 0, msDome_ = 0, msRender_ = 0, msTrace_ = 0, msShade_ = 0, msShadow_ = 0;
    float     msBvhWall_ = 0, msBvhAlloc_ = 0; // last full build: host wall time, and its cudaMalloc share
    std::vector<uint64_t> waveRays_;       // CL_PROFILE_STAGES: closest-hit rays of each wave of the last render
    unsigned long long    waveRaysSeen_ = 0;
    cudaEvent_t evA_ = nullptr, evB_ = nullptr, evS_[6] = {};

    // Guiding.
    std::unique_ptr<GuideNet> guide_;
    cl_guide_config           guideCfg_{};
    DevBuf                    lobes_, hist_, rec_;
    uint32_t                  recStride_ = 0, recCap_ = 0, histSlots_ = 0, histDepth_ = 0;
    float                     boxMin_[3] = {0, 0, 0}, boxScale_ = 1.0f;
    int                       inferBlocks_ = 0;
    uint64_t                  guideSamples_ = 0, guideRecordsLast_ = 0, guideInferred_ = 0;
    double                    guideLoss_ = 0.0;
    float                     msTrain_ = 0.0f, msInfer_ = 0.0f;

    // Radiance cache.
    std::unique_ptr<CacheNet>  cache_;
    cl_radiance_cache_config   cacheCfg_{};
    DevBuf                     cacheL_, cacheEnc_, cacheEncIdx_, cacheHist_, cacheRec_;
    uint32_t                   cacheRecCap_ = 0, cacheHistDepth_ = 0;
    int                        cacheEncodeBlocks_ = 0, cacheMlpBlocks_ = 0;
    uint64_t                   cacheSamples_ = 0, cacheRecordsLast_ = 0, cacheQueries_ = 0;
    double                     cacheLoss_ = 0.0;
    float                      msCacheTrain_ = 0.0f;
};

} // namespace clb
